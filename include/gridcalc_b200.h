/* gridcalc_b200 — C ABI of the B200 (sm_100a) periodic-grid operator and
 * time-stepping library.
 *
 * The reference gridcalc 0.15.1 is a header-only C++17 library with no FFI:
 * its interface is templated free functions over core::Field<double>.  Each
 * entry point below replaces one of those functions (cited per declaration)
 * with a call over raw device buffers, so a C, C++, ctypes or any FFI caller
 * can bind it; the C++ drop-in headers in grid-calculus_b200/include/gridcalc
 * rebuild the reference signatures on top of it.
 *
 * Conventions
 *  - Buffers are DEVICE pointers owned by the caller, laid out i-fastest:
 *    cell (i, j, k) at i + Nx*(j + Ny*k) (reference core/Grid.hpp:132-137).
 *    Vector fields are three consecutive planes (x, y, z components, N
 *    values each), the coalescing-friendly layout; the C++ drop-in converts
 *    from the reference's interleaved Field<Vec3d>.
 *  - dtype selects the storage type of every field argument of a call:
 *    GC_F64 (double) or GC_F32 (float).  F64 arithmetic follows the
 *    reference tap order without FMA contraction; F32 computes stencils in
 *    float and every integral (integrate, evaluate, mass, energy) in double.
 *  - Work is stream-ordered with the caller's stream.  Calls that return a host
 *    scalar or report a data-dependent error (integrate, evaluate, the D > 0
 *    check, the CFL check of diffuse_fvm) synchronise that stream; the
 *    others return after enqueueing.  gc_synchronize() waits for all work.
 *  - Scratch is allocated on first use and kept by the context (cudaMalloc
 *    happens only when a call needs more than the context already holds).
 *  - No entry point throws.  A non-GC_OK status comes with a message from
 *    gc_last_error() (thread-local) that carries the reference's wording:
 *    "axis x|y|z" for extents, "flat index" for D <= 0, "solve::diffuse" for
 *    CFL, "k1".."k4" never arise (device RHS functors cannot change grids).
 *  - One context per host thread; a context is not thread-safe.
 */
#ifndef GRIDCALC_B200_H
#define GRIDCALC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GC_API __attribute__((visibility("default")))
#else
#define GC_API
#endif

typedef enum gc_status {
  GC_OK = 0,
  GC_ERR_INVALID_ARG = 1,   /* std::invalid_argument in the reference */
  GC_ERR_AXIS_EXTENT = 2,   /* diff/detail/PreconditionAxisExtent.hpp:64-79 */
  GC_ERR_GRID_MISMATCH = 3, /* solve/detail/RhsGridCheck.hpp:42-64 */
  GC_ERR_NONPOSITIVE_D = 4, /* fvm/CellLaplacian.hpp:100-109 */
  GC_ERR_CFL = 5,           /* solve/Diffusion.hpp:45-59 */
  GC_ERR_CUDA = 6,          /* a CUDA runtime call failed */
  GC_ERR_TIMEOUT = 7,       /* a bounded device-side wait gave up */
  GC_ERR_NONFINITE = 8,     /* a non-finite value was detected in the state */
  GC_ERR_UNSUPPORTED = 9,   /* (order, dtype, shape) combination not built */
  GC_ERR_IO = 10            /* a file could not be opened, read or written, or failed its checks */
} gc_status;

typedef enum gc_dtype { GC_F64 = 0, GC_F32 = 1 } gc_dtype;

/* func::Pairwise / func::Kahan (func/Integrate.hpp:43,52). */
typedef enum gc_sum { GC_SUM_PAIRWISE = 0, GC_SUM_KAHAN = 1 } gc_sum;

/* solve::ExplicitEuler / solve::RK4 tags (solve/ExplicitEuler.hpp:37-41,
 * solve/RK4.hpp:30-35). */
typedef enum gc_integrator { GC_EXPLICIT_EULER = 0, GC_RK4 = 1 } gc_integrator;

/* core::Grid (core/Grid.hpp:28-148): extents and per-axis cell size. */
typedef struct gc_grid {
  int32_t nx, ny, nz;
  double hx, hy, hz;
} gc_grid;

typedef struct gc_context gc_context;

/* ---- context, errors, memory ------------------------------------------- */

/* Creates a context on `device` for callers working on `stream` (a
 * cudaStream_t; NULL = the default stream).  The context runs its kernels on
 * a stream of its own (so that step sequences can be captured into CUDA
 * graphs) and orders every call after prior work on `stream` and later work
 * on `stream` after the call.  It owns its scratch (RK stage buffers,
 * reduction partials, captured graphs). */
GC_API gc_status gc_context_create(gc_context** out, int device, void* stream);
GC_API gc_status gc_context_destroy(gc_context* ctx);
/* Context switches (no reference counterpart).
 *   GC_OPT_CLUSTER_STEPPING (default 0): 1 makes gc_ch_integrate advance a
 *     2-D grid whose whole state fits in the shared memory of one
 *     thread-block cluster (up to 16 CTAs; about 240 x 240 doubles with RK4)
 *     in a single cluster-resident launch for all its steps.  Off by
 *     default: on B200 the fused step kernel below is faster at every such
 *     size (128^2: 9.2 against 13.1 us per RK4 step).  Same values, bit for
 *     bit in double.
 *   GC_OPT_FUSED_STEP (default 1): gc_ch_integrate runs each RK4 step of a
 *     2-D double grid at order 2, and of a 2-D float grid at order 2 or 4,
 *     as one fused kernel (all four stages on a tile with a halo of 8R cells
 *     in shared memory; psi read and psi' written once per step); 0 uses
 *     the four stage kernels.  Same values, bit for bit, in double; in
 *     float the two may differ in rounding. */
typedef enum gc_option { GC_OPT_CLUSTER_STEPPING = 0, GC_OPT_FUSED_STEP = 1 } gc_option;
GC_API gc_status gc_context_set_option(gc_context* ctx, int32_t option, int32_t value);
GC_API gc_status gc_synchronize(gc_context* ctx);
/* Failure-detection self-test (no reference counterpart): launches one
 * thread that waits on a device flag nothing sets, gives up after
 * budget_cycles (at most 4e9, about 2 s) and records GC_ERR_TIMEOUT exactly
 * as a bounded TMA wait does; the next gc_synchronize reports it and clears
 * it, and the context stays usable. */
GC_API gc_status gc_selftest_bounded_wait(gc_context* ctx, int64_t budget_cycles);
GC_API const char* gc_last_error(void);
GC_API const char* gc_status_string(gc_status s);
/* gridcalc::version() (include/gridcalc/version.hpp.in:16-18). */
GC_API const char* gc_version(void);
/* Device memory helpers for callers without a CUDA runtime binding. */
GC_API gc_status gc_malloc(gc_context* ctx, size_t bytes, void** dev);
GC_API gc_status gc_free(gc_context* ctx, void* dev);
GC_API gc_status gc_memcpy_h2d(gc_context* ctx, void* dev, const void* host, size_t bytes);
GC_API gc_status gc_memcpy_d2h(gc_context* ctx, void* host, const void* dev, size_t bytes);

/* ---- operators (diff::, fvm::) ------------------------------------------ */

/* diff::laplacian<Order> (diff/Laplacian.hpp:44-75); order 2, 4 or 6. */
GC_API gc_status gc_laplacian(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                              const void* in, void* out);
/* diff::gradient<Order>, scalar -> vector (diff/Gradient.hpp:43-74). */
GC_API gc_status gc_gradient(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                             const void* in, void* out3);
/* diff::divergence<Order>, vector -> scalar (diff/Divergence.hpp:43-74). */
GC_API gc_status gc_divergence(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                               const void* in3, void* out);
/* diff::gradient<Order>, Vec3d -> Mat3d (diff/Gradient.hpp:100-137).  in3 is
 * three planes (x, y, z components); out9 is nine planes, plane 3*row + col
 * holding M(row, col) = d_col v_row. */
GC_API gc_status gc_gradient_vec(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                                 const void* in3, void* out9);
/* diff::divergence<Order>, Mat3d -> Vec3d (diff/Divergence.hpp:100-135):
 * (div M)_row = sum over col of d_col M(row, col), same plane layouts. */
GC_API gc_status gc_divergence_mat(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                                   const void* in9, void* out3);
/* diff::biharmonic<Order> / diff::d4 (diff/Biharmonic.hpp:48-119). */
GC_API gc_status gc_biharmonic(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order,
                               const void* in, void* out);

/* diff::detail::mixedDerivative<ax, ay, az, Order> (diff/detail/MultiIndexDerivative.hpp:96-137):
 * d^(ax+ay+az) in / dx^ax dy^ay dz^az, each count 0..4.  The reference's 31
 * named partials forward here: dxx dyy dzz dxy dxz dyz (diff/MixedPartial.hpp),
 * d3dx3 ... d3dxdydz (diff/ThirdOrder.hpp), d4dx4 ... d4dxdydz2
 * (diff/FourthOrder.hpp).  Orders 2 and 4 as the reference, 6 added.  Each
 * axis is checked against its own stencil radius (0 for a count of 0). */
GC_API gc_status gc_partial(gc_context* ctx, const gc_grid* g, gc_dtype dt, int order, int ax, int ay, int az,
                            const void* in, void* out);
/* fvm::cellLaplacian (fvm/CellLaplacian.hpp:91-143).  Checks D > 0 first;
 * on violation returns GC_ERR_NONPOSITIVE_D and the first flat index in
 * *bad_index (may be NULL). */
GC_API gc_status gc_cell_laplacian(gc_context* ctx, const gc_grid* g, gc_dtype dt,
                                   const void* psi, const void* D, void* out,
                                   int64_t* bad_index);

/* ---- integrals (func::) -------------------------------------------------- */

/* func::integrate(field, Pairwise|Kahan) (func/Integrate.hpp:116-135):
 * cell volume times the sum.  GC_SUM_PAIRWISE reproduces the reference's
 * recursive pairwise tree (base case 64) exactly, so F64 results are
 * bit-identical; GC_SUM_KAHAN is a deterministic compensated parallel sum. */
GC_API gc_status gc_integrate(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* in,
                              gc_sum sum, double* result);

/* Allocation-free variant of gc_integrate with the Pairwise tag (no
 * counterpart in the reference, which has no device memory at all).  For
 * callers that cannot allocate device memory: applications whose device
 * memory belongs entirely to another allocator, plug-in hosts that only
 * hand over buffers, loops that forbid allocation once running.  It needs
 * no context: it runs on `stream` (a cudaStream_t, NULL = default stream)
 * and writes cell volume times the exact pairwise sum (bit-identical to
 * gc_integrate) to the device double *result_dev, stream-ordered, without
 * synchronising.  Its scratch is a fixed 525 KB device array inside the
 * library, held by every GPU that loads it until exit, which limits the
 * field to 2^29 cells (larger fields get GC_ERR_INVALID_ARG).  All calls
 * share that array: calls that overlap on the GPU race, so keep them on one
 * stream.  The first call on each device (with that device current) looks
 * up the array's device address and keeps it for the life of the process;
 * make it before any stream capture, and do not reset the device
 * (cudaDeviceReset) after it, since the kept address would then be stale. */
GC_API gc_status gc_integrate_noalloc(const gc_grid* g, gc_dtype dt, const void* in,
                                      double* result_dev, void* stream);

/* Integrands for func::evaluate (func/Functional.hpp:88-148), one per
 * use of the reference's callable forms on the hot path. */
typedef enum gc_integrand_kind {
  GC_INTEGRAND_PSI = 0,             /* f(psi) = psi        (cahn_hilliard.hpp:111) */
  GC_INTEGRAND_PSI_SQUARED = 1,     /* f(psi) = psi^2      (heterogeneous_diffusion.hpp:82) */
  GC_INTEGRAND_CH_FREE_ENERGY = 2,  /* -psi^2/2 + psi^4/4 + kappa/2 |grad psi|^2 (cahn_hilliard.hpp:64-68) */
  GC_INTEGRAND_GRAD_SQUARED = 3     /* |grad psi|^2        (cahn_hilliard.hpp:73-77) */
} gc_integrand_kind;

typedef struct gc_integrand {
  int32_t kind;  /* gc_integrand_kind */
  double kappa;  /* GC_INTEGRAND_CH_FREE_ENERGY only */
} gc_integrand;

/* func::evaluate(psi, f, tag): the integrand is formed on the device from
 * psi and its order-2 gradient (the reference's default) and reduced in FP64,
 * in one pass over psi (the integrand runs as a built-in program of
 * gc_evaluate_program below, with the reference expression's operations in
 * its order). */
GC_API gc_status gc_evaluate(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* psi,
                             const gc_integrand* f, gc_sum sum, double* result);

/* General integrands.  func::evaluate (func/Functional.hpp:88-148 for a
 * scalar psi, :183-220 for a Vec3d field u) calls a host callable per cell
 * whose arity picks the derivative fields it receives.  Across the C ABI the
 * callable is a straight-line program over double registers r[0..31]: each
 * instruction writes r[dst] from r[a], r[b], a constant or an input, with
 * correctly rounded + - * / and sqrt, so a program that performs the
 * callable's operations in the callable's order yields the same integrand,
 * bit for bit.  The program's value is r[dst] of its last instruction.
 *
 * Inputs (order-2 derivatives, the reference's default), by arity:
 *   scalar (components 1): arity 1: GC_IN_PSI; 2 adds GC_IN_GRAD_X..Z;
 *     3 adds GC_IN_LAP; 4 adds GC_IN_BIH.
 *   vector (components 3): arity 1: GC_IN_U_X..Z; 2 adds GC_IN_DU + 3*row + col,
 *     the rank-2 gradient M(row, col) = d_col u_row (diff/Gradient.hpp:100-137). */
#define GC_PROGRAM_MAX_INSTR 128
#define GC_PROGRAM_REGS 32

typedef enum gc_opcode {
  GC_OPC_CONST = 0,  /* r[dst] = value */
  GC_OPC_INPUT = 1,  /* r[dst] = input number a */
  GC_OPC_ADD = 2,    /* r[dst] = r[a] + r[b] */
  GC_OPC_SUB = 3,    /* r[dst] = r[a] - r[b] */
  GC_OPC_MUL = 4,    /* r[dst] = r[a] * r[b] */
  GC_OPC_DIV = 5,    /* r[dst] = r[a] / r[b] */
  GC_OPC_NEG = 6,    /* r[dst] = -r[a] */
  GC_OPC_ABS = 7,    /* r[dst] = |r[a]| */
  GC_OPC_SQRT = 8,   /* r[dst] = sqrt(r[a]) */
  GC_OPC_MIN = 9,    /* r[dst] = std::min(r[a], r[b]) = r[b] < r[a] ? r[b] : r[a] */
  GC_OPC_MAX = 10    /* r[dst] = std::max(r[a], r[b]) = r[a] < r[b] ? r[b] : r[a] */
} gc_opcode;

enum {
  GC_IN_PSI = 0, GC_IN_GRAD_X = 1, GC_IN_GRAD_Y = 2, GC_IN_GRAD_Z = 3, GC_IN_LAP = 4, GC_IN_BIH = 5,
  GC_IN_U_X = 0, GC_IN_U_Y = 1, GC_IN_U_Z = 2, GC_IN_DU = 3
};

typedef struct gc_instr {
  int16_t op, dst, a, b;  /* gc_opcode; register or input numbers (unused ones 0) */
  double value;           /* GC_OPC_CONST only */
} gc_instr;

typedef struct gc_program {
  int32_t components;  /* 1: scalar psi; 3: vector u (three planes) */
  int32_t arity;       /* 1..4 (scalar) or 1..2 (vector), as the callable's */
  int32_t n_instr;     /* 1..GC_PROGRAM_MAX_INSTR */
  int32_t reserved;    /* 0 */
  gc_instr instr[GC_PROGRAM_MAX_INSTR];
} gc_program;

/* func::evaluate(field, f, tag) for a program f.  The derivative fields of
 * f's arity are checked against the axis extents in the reference's order
 * (gradient, Laplacian, biharmonic), the integrand is formed on the device
 * and reduced like gc_integrate.  A malformed program (bad opcode, register
 * read before it is written, input beyond the arity) is GC_ERR_INVALID_ARG. */
GC_API gc_status gc_evaluate_program(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* field,
                                     const gc_program* f, gc_sum sum, double* result);
/* The CUDA source gc_evaluate_program compiles for f (NVRTC, sm_100a), for
 * inspection: copies at most cap - 1 characters and a terminating NUL into
 * buf and returns the full size including the NUL (0 for a malformed
 * program).  Each distinct source is compiled once per process and device. */
GC_API size_t gc_program_source(const gc_program* f, gc_dtype dt, char* buf, size_t cap);
/* The program gc_evaluate runs for a named integrand (the reference
 * expression's operations in its order; kappa enters as the constant
 * 0.5 * kappa).  No counterpart in the reference; no GPU work. */
GC_API gc_status gc_integrand_program(const gc_integrand* f, gc_program* out);

/* Non-finite detection (no counterpart in the reference, which has no such
 * check): scans `components` planes of a device field for a NaN or an
 * infinity.  All finite: GC_OK and *first_bad = -1.  Otherwise
 * GC_ERR_NONFINITE, *first_bad = the first flat index, and the message names
 * the value, its component and its cell.  Run it after a batch of steps or
 * before a snapshot to catch a blown-up trajectory. */
GC_API gc_status gc_check_finite(gc_context* ctx, const gc_grid* g, gc_dtype dt, int32_t components,
                                 const void* field, int64_t* first_bad);

/* ---- time integration (solve::) ----------------------------------------- */

/* Cahn-Hilliard right-hand side M lap(-psi + psi^3 - kappa lap psi)
 * (examples/common/cahn_hilliard.hpp:38-59) at Laplacian order 2, 4 or 6. */
typedef struct gc_ch_params {
  double mobility;
  double kappa;
  int32_t order;
} gc_ch_params;

/* One evaluation of the Cahn-Hilliard RHS (computeRhs). */
GC_API gc_status gc_ch_rhs(gc_context* ctx, const gc_grid* g, gc_dtype dt,
                           const gc_ch_params* p, const void* psi, void* out);

/* solve::integrate(psi, computeRhs, dt, n_steps, RK4|ExplicitEuler)
 * (solve/RK4.hpp:99-154, solve/ExplicitEuler.hpp:79-112) with the
 * Cahn-Hilliard RHS, psi advanced in place.  RK4 runs four fused stage
 * kernels per step (each reads and writes every field once); the steps are
 * replayed from a captured CUDA graph (a 2-D double grid at order 2, or a
 * 2-D float grid at order 2 or 4, runs one fused kernel per step instead,
 * GC_OPT_FUSED_STEP).  With
 * GC_OPT_CLUSTER_STEPPING on, a 2-D grid whose state fits in one
 * thread-block cluster's shared memory (gc_ch_cluster_ctas > 0) runs all
 * n_steps in one cluster-resident launch. */
GC_API gc_status gc_ch_integrate(gc_context* ctx, const gc_grid* g, gc_dtype dt,
                                 const gc_ch_params* p, void* psi, double dt_step,
                                 int n_steps, gc_integrator integrator);
/* CTAs of the cluster that gc_ch_integrate uses for this 2-D grid, storage
 * type, Laplacian order and integrator (one slab of rows per CTA, the
 * slab's psi, stage fields and halos in that CTA's shared memory); 0 when
 * the state does not fit and the per-stage kernels run.  No GPU work. */
GC_API int32_t gc_ch_cluster_ctas(const gc_grid* g, gc_dtype dt, int32_t order, gc_integrator integrator);

/* RKC2 (damped second-order Runge-Kutta-Chebyshev, eps = 2/13) with
 * `stages` stages (2..64): n_steps steps of dt_step, psi in place, same RHS
 * as gc_ch_integrate.  No reference counterpart (the reference offers
 * Euler and RK4); it is the base step of the learned coarse step.  Stable
 * for dt_step * lambda_max <= gc_rkc_stability_bound(stages) (~0.65 s^2),
 * lambda_max the spectral radius of the linearised RHS. */
GC_API gc_status gc_ch_rkc(gc_context* ctx, const gc_grid* g, gc_dtype dt, const gc_ch_params* p, void* psi,
                           double dt_step, int32_t n_steps, int32_t stages);
GC_API double gc_rkc_stability_bound(int32_t stages);

/* makeRandomIc (examples/common/cahn_hilliard.hpp:85-103): fills the HOST
 * buffer out (nx*ny*nz doubles, i fastest) with one draw per cell, in flat
 * index order, of std::uniform_real_distribution<double>(-amplitude,
 * amplitude) over std::mt19937_64(seed) -- the bytes the reference's build
 * produces with libstdc++.  subtract_mean != 0 then subtracts the draws' mean
 * (sequential sum / n) as the reference does; 0 keeps the raw draws
 * (c = 0 plus i.i.d. uniform noise).  No GPU work. */
GC_API gc_status gc_random_ic(const gc_grid* g, uint64_t seed, double amplitude, int32_t subtract_mean,
                              double* out);

/* solve::diffuse(psi, double D, dt, n_steps, tag) (solve/Diffusion.hpp:89-112):
 * constant-D heat equation with the order-2 Laplacian and the tag's CFL check. */
GC_API gc_status gc_diffuse(gc_context* ctx, const gc_grid* g, gc_dtype dt, void* psi,
                            double D, double dt_step, int n_steps, gc_integrator integrator);

/* solve::diffuse(psi, Field D, dt, n_steps, tag) (solve/Diffusion.hpp:161-216):
 * FVM heat equation.  The largest harmonic face D is found on the device,
 * the CFL check and the D > 0 check run once before the first step. */
GC_API gc_status gc_diffuse_fvm(gc_context* ctx, const gc_grid* g, gc_dtype dt, void* psi,
                                const void* D, double dt_step, int n_steps,
                                gc_integrator integrator, int64_t* bad_index);

/* Largest harmonic-mean face D over +x/+y/+z faces (solve/Diffusion.hpp:187-207). */
GC_API gc_status gc_d_max_face(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* D,
                               double* result);

/* ---- batched Cahn-Hilliard ensemble --------------------------------------
 * No reference counterpart as one call: it replaces a loop over independent
 * solve::integrate(psi_i, computeRhs, dt_i, n, RK4{}) runs
 * (solve/RK4.hpp:99-154, examples/common/cahn_hilliard.hpp:38-59), each
 * member on its own 2-D periodic grid with h = 1 and its own mobility, kappa
 * and time step, all at one Laplacian order and storage type.  Members'
 * fields are packed in one device buffer: member i occupies elements
 * [offsets[i], offsets[i] + nx*ny) (i fastest) of gc_ch_batch_state(). */
typedef struct gc_ch_member {
  int32_t nx, ny;
  double mobility, kappa, dt;
} gc_ch_member;

typedef struct gc_ch_batch gc_ch_batch;

GC_API gc_status gc_ch_batch_create(gc_context* ctx, int32_t n, const gc_ch_member* members,
                                    int32_t order, gc_dtype dt, gc_ch_batch** out);
GC_API gc_status gc_ch_batch_destroy(gc_ch_batch* b);
/* n + 1 element offsets of the members in the packed state. */
GC_API gc_status gc_ch_batch_offsets(gc_ch_batch* b, int64_t* offsets);
/* Device pointer to the packed state (fill it with gc_memcpy_h2d). */
GC_API gc_status gc_ch_batch_state(gc_ch_batch* b, void** dev);
/* Advances every member by n_steps RK4 steps; steps replay from a captured
 * CUDA graph.  With the fused shape (GC_BATCH_FUSED, the default at
 * Laplacian orders 2 and 4) one persistent launch per step runs all four
 * stages of every (member, tile) work item in shared memory; the other
 * shapes are four persistent launches per step, one per stage. */
GC_API gc_status gc_ch_batch_run(gc_ch_batch* b, int32_t n_steps);
/* Tile shapes: 0..3 the stage kernels' tiles (32x16x4, 64x8x4, 64x16x4,
 * 64x32x8: threads in x, output rows, thread rows), GC_BATCH_FUSED the fused
 * four-stage kernel (64 x 32 output tiles for float, 64 x 16 for double;
 * orders 2 and 4 only, GC_ERR_UNSUPPORTED at order 6).  Results do not
 * depend on the shape in double; in float they may differ in rounding. */
#define GC_BATCH_FUSED 4
GC_API gc_status gc_ch_batch_set_shape(gc_ch_batch* b, int32_t shape);
/* Per-member mass and free energy (reference convention, order-2 gradient),
 * accumulated in double with compensated sums in a fixed order. */
GC_API gc_status gc_ch_batch_diagnostics(gc_ch_batch* b, double* mass, double* free_energy);
/* Times each tile shape that fits the order (steps_per_trial steps each,
 * state restored afterwards) and keeps the fastest; with cache_path, reuses
 * or records the choice in a JSON file keyed by device and ensemble.  A JSON
 * report of the trials is written to report. */
GC_API gc_status gc_ch_batch_autotune(gc_ch_batch* b, int32_t steps_per_trial, const char* cache_path,
                                      char* report, size_t report_len);

/* ---- learned coarse-step corrector ---------------------------------------
 * No reference counterpart.  A 6-layer periodic 3x3 CNN (32 channels, GELU
 * in tanh form, BF16 weights and activations, FP32 accumulation on the
 * tensor cores) maps a 2-D Cahn-Hilliard field c to a zero-mean correction
 * delta so that the coarse step -- c + delta, or B(c) + delta over a base
 * step B (see gc_corrector_set_base) -- approximates fine_per_coarse plain
 * RK4 steps.  Parameters are FP32 masters, per layer W[9 taps][32 in][32 out]
 * then b[32], tap t at offset (t / 3 - 1, t % 3 - 1) in (y, x).  Input
 * channels: c, u = (B(c) - c) / rms and e = est / rms with est = (B(c) - c)
 * / Dt - (f(c) + f(B(c))) / 2 (u = e = 0 without a base step);
 * delta = s_out rho (z6 - mean z6), z6 the last layer's channel 0, rho =
 * Dt rms(est) per sample (1 without a base step). */
typedef struct gc_corrector gc_corrector;

typedef struct gc_corrector_policy {
  double dt_fine;           /* fine RK4 step (the plain method's dt) */
  int32_t fine_per_coarse;  /* fine steps one coarse step replaces */
  double residual_tol;      /* accept when the trapezoid residual is at most this */
  double energy_tol;        /* accept when F rises by at most energy_tol + energy_rtol |F| */
  double energy_rtol;
  int32_t try_base;         /* with a base step: a rejected proposal B(c) + delta is followed by
                               the same test on B(c) alone before falling back to plain RK4 */
} gc_corrector_policy;

typedef struct gc_corrector_stats {
  int64_t accepted;           /* coarse steps taken by the network */
  int64_t fallbacks;          /* coarse steps taken by plain RK4 instead */
  int64_t rejected_energy;    /* fallbacks whose proposal raised F beyond the tolerance */
  int64_t rejected_residual;  /* fallbacks whose proposal's residual exceeded residual_tol */
  int64_t accepted_base;      /* coarse steps taken by the base step alone (try_base) */
  double last_residual;
} gc_corrector_stats;

GC_API gc_status gc_corrector_create(gc_context* ctx, int32_t height, int32_t width, int32_t max_batch,
                                     gc_corrector** out);
GC_API gc_status gc_corrector_destroy(gc_corrector* c);
GC_API int32_t gc_corrector_num_params(void);
GC_API gc_status gc_corrector_set_params(gc_corrector* c, const float* host, int32_t n, float s_out);
/* Base step: one gc_ch_rkc step of dt_coarse with `stages` stages and the
 * RHS p on unit cell spacing.  With it, the coarse step is B(c) + delta and
 * the network also sees the base step's increment and error indicator;
 * NULL p turns it off (coarse step c + delta). */
GC_API gc_status gc_corrector_set_base(gc_corrector* c, const gc_ch_params* p, double dt_coarse, int32_t stages);
/* normalized != 0: the training loss weights each sample by 1 / mean((target
 * - s)^2), s = B(c) with a base step else c, so that small (late-time) steps
 * count as much as large ones. */
GC_API gc_status gc_corrector_set_loss(gc_corrector* c, int32_t normalized);
GC_API gc_status gc_corrector_get_params(gc_corrector* c, float* host, int32_t n);
/* The coarse-step increment (B(c) - c + delta, or delta without a base
 * step) for `batch` fields (batch x height x width, dtype F32 or F64) into
 * delta_out (device, float). */
GC_API gc_status gc_corrector_forward(gc_corrector* c, int32_t batch, gc_dtype dt, const void* cin,
                                      float* delta_out);
/* Gradient w.r.t. all parameters (host, num_params floats; parameters
 * unchanged) of the loss sum_b sum_p (s_b + delta_b - target_b)^2 / (N den_b):
 * s = B(c) with a base step else c, N = batch x height x width, den_b =
 * mean((target_b - s_b)^2) with the normalised loss else 1.  cin and target
 * are device fields of dtype dt. */
GC_API gc_status gc_corrector_gradient(gc_corrector* c, int32_t batch, gc_dtype dt, const void* cin,
                                       const void* target, float* grad_host, double* loss);
/* One Adam step (beta 0.9 / 0.999) on that loss. */
GC_API gc_status gc_corrector_train_step(gc_corrector* c, int32_t batch, gc_dtype dt, const void* cin,
                                         const void* target, float lr, double* loss);
/* Learned coarse steps on one double field with the plain-RK4 fallback
 * (and, with pol->try_base, the base step alone as the first fallback).
 * rejected_energy / rejected_residual count the network's rejected
 * proposals by cause (one can fail both); accepted_base of them were taken
 * by the base step alone, fallbacks by plain RK4. */
GC_API gc_status gc_corrector_advance(gc_corrector* c, const gc_grid* g, const gc_ch_params* cp, double* psi,
                                      int32_t n_coarse, const gc_corrector_policy* pol,
                                      gc_corrector_stats* stats);

/* ---- spectral derivatives (spectral/Derivatives.hpp, Wavenumbers.hpp) ----
 * FFT-based derivatives of a periodic double field: forward real-to-complex
 * transform, the derivative's multiplier on the half spectrum, inverse
 * transform.  Wavenumbers k = 2 pi n / (N h); an odd derivative count along
 * an axis of even extent zeroes that axis's Nyquist mode.  Double fields
 * only; Nx = 1 with another axis longer than 1 is GC_ERR_UNSUPPORTED.
 * Agrees with the reference's PocketFFT path to rounding. */
/* spectral::partial<ax, ay, az> (spectral/Derivatives.hpp:78-134), counts 0..8. */
GC_API gc_status gc_spectral_partial(gc_context* ctx, const gc_grid* g, gc_dtype dt, int ax, int ay, int az,
                                     const void* in, void* out);
/* spectral::laplacian (:144-172) and spectral::biharmonic (:175-204). */
GC_API gc_status gc_spectral_laplacian(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* in, void* out);
GC_API gc_status gc_spectral_biharmonic(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* in, void* out);
/* spectral::gradient (:207-240): three planes out. */
GC_API gc_status gc_spectral_gradient(gc_context* ctx, const gc_grid* g, gc_dtype dt, const void* in, void* out3);

/* ---- snapshot output and checkpoint / resume ---------------------------- */

typedef enum gc_vtk_encoding { GC_VTK_ASCII = 0, GC_VTK_BINARY = 1 } gc_vtk_encoding;

/* gridcalc::examples::writeVtkStructuredPoints (examples/common/vtk_writer.hpp:34-66):
 * legacy VTK 3.0 STRUCTURED_POINTS with one SCALARS array of doubles, i
 * fastest.  GC_VTK_ASCII writes the reference's bytes exactly (17
 * significant digits per value); GC_VTK_BINARY the same header with
 * big-endian doubles.  host: the field in host memory (dt values, float
 * written as double).  Needs no device. */
GC_API gc_status gc_write_vtk(const gc_grid* g, gc_dtype dt, const void* host, const char* path,
                              const char* field_name, gc_vtk_encoding enc);

/* Checkpoint file: an 80-byte little-endian header (magic "GCB200CK",
 * version 2, dtype, nx ny nz, components, hx hy hz, data bytes, metadata
 * bytes, 64-bit checksum of the header, the metadata and the data), the
 * metadata (e.g. JSON: step, time, parameters), then `components` planes of
 * the field, i fastest.  Written under a temporary name and renamed.  Version
 * 1 files (checksum of the data only) are read as well.  Needs no device. */
GC_API gc_status gc_write_checkpoint(const gc_grid* g, gc_dtype dt, int32_t components, const void* host,
                                     const char* path, const char* meta_json);
/* The header of a checkpoint: grid, dtype, components and metadata length. */
GC_API gc_status gc_checkpoint_info(const char* path, gc_grid* g, gc_dtype* dt, int32_t* components,
                                    size_t* meta_len);
/* Reads the field into host memory (host_bytes >= its size) and the
 * metadata into meta (NUL-terminated, at most meta_cap - 1 characters; may
 * be NULL).  A missing, truncated or corrupt file (bad magic, inconsistent
 * header, checksum mismatch) is GC_ERR_IO. */
GC_API gc_status gc_read_checkpoint(const char* path, void* host, size_t host_bytes, char* meta, size_t meta_cap);
/* The same into a device buffer, ordered on the context's stream (returns
 * after the copy). */
GC_API gc_status gc_load_checkpoint(gc_context* ctx, const char* path, void* field, size_t field_bytes, char* meta,
                                    size_t meta_cap);

/* Snapshots of device fields that do not stall the computation: each call
 * copies the field device-to-device on the context's stream into one of
 * `depth` slots (so later work may overwrite the field at once), a copy
 * stream moves the slot to pinned host memory while later work runs, and a
 * writer thread writes the file.  A call waits only when all slots still
 * hold unwritten snapshots.  One thread at a time per snapshotter. */
typedef struct gc_snapshotter gc_snapshotter;
GC_API gc_status gc_snapshotter_create(gc_context* ctx, int32_t depth, gc_snapshotter** out);
GC_API gc_status gc_snapshot_vtk(gc_snapshotter* s, const gc_grid* g, gc_dtype dt, const void* field,
                                 const char* path, const char* field_name, gc_vtk_encoding enc);
GC_API gc_status gc_snapshot_checkpoint(gc_snapshotter* s, const gc_grid* g, gc_dtype dt, int32_t components,
                                        const void* field, const char* path, const char* meta_json);
/* Waits until every queued file is written; returns the first write error. */
GC_API gc_status gc_snapshotter_flush(gc_snapshotter* s);
/* Flushes, stops the writer thread and frees the slots. */
GC_API gc_status gc_snapshotter_destroy(gc_snapshotter* s);

#ifdef __cplusplus
}
#endif
#endif /* GRIDCALC_B200_H */
