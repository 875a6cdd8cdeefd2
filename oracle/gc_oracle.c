/* CPU oracle (test infrastructure only; see gc_oracle.h).
 *
 * Plain-C restatement of the reference gridcalc hot path.  Each routine
 * cites the reference file:line it restates and keeps the reference's
 * arithmetic order: per-axis tap accumulation from 0.0 in offset order,
 * axis terms combined left to right, no FMA (compile with
 * -ffp-contract=off).  Periodic wrap uses per-axis neighbour tables instead
 * of the reference's per-access ((i % N) + N) % N; the values read are the
 * same.
 */
#include "gc_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static char g_err[512];

const char* oc_last_error(void) { return g_err; }

/* ---- stencil tables: stencil/CentralDifference.hpp:41-74,
 * FirstDerivative.hpp:51-86, ThirdDerivative.hpp:49-84,
 * FourthDerivative.hpp:49-83; order 6 added (no reference counterpart). */
int oc_weights(int kind, int order, double* w) {
  if (kind == 2 && order == 2) { w[0] = 1.0; w[1] = -2.0; w[2] = 1.0; return 1; }
  if (kind == 2 && order == 4) {
    w[0] = -1.0 / 12.0; w[1] = 4.0 / 3.0; w[2] = -5.0 / 2.0; w[3] = 4.0 / 3.0; w[4] = -1.0 / 12.0;
    return 2;
  }
  if (kind == 2 && order == 6) {
    w[0] = 1.0 / 90.0; w[1] = -3.0 / 20.0; w[2] = 3.0 / 2.0; w[3] = -49.0 / 18.0;
    w[4] = 3.0 / 2.0; w[5] = -3.0 / 20.0; w[6] = 1.0 / 90.0;
    return 3;
  }
  if (kind == 1 && order == 2) { w[0] = -0.5; w[1] = 0.0; w[2] = 0.5; return 1; }
  if (kind == 1 && order == 4) {
    w[0] = 1.0 / 12.0; w[1] = -2.0 / 3.0; w[2] = 0.0; w[3] = 2.0 / 3.0; w[4] = -1.0 / 12.0;
    return 2;
  }
  if (kind == 1 && order == 6) {
    w[0] = -1.0 / 60.0; w[1] = 3.0 / 20.0; w[2] = -3.0 / 4.0; w[3] = 0.0;
    w[4] = 3.0 / 4.0; w[5] = -3.0 / 20.0; w[6] = 1.0 / 60.0;
    return 3;
  }
  if (kind == 3 && order == 2) {
    w[0] = -1.0 / 2.0; w[1] = 1.0; w[2] = 0.0; w[3] = -1.0; w[4] = 1.0 / 2.0;
    return 2;
  }
  if (kind == 3 && order == 4) {
    w[0] = 1.0 / 8.0; w[1] = -1.0; w[2] = 13.0 / 8.0; w[3] = 0.0;
    w[4] = -13.0 / 8.0; w[5] = 1.0; w[6] = -1.0 / 8.0;
    return 3;
  }
  if (kind == 3 && order == 6) {
    w[0] = -7.0 / 240.0; w[1] = 3.0 / 10.0; w[2] = -169.0 / 120.0; w[3] = 61.0 / 30.0; w[4] = 0.0;
    w[5] = -61.0 / 30.0; w[6] = 169.0 / 120.0; w[7] = -3.0 / 10.0; w[8] = 7.0 / 240.0;
    return 4;
  }
  if (kind == 4 && order == 2) {
    w[0] = 1.0; w[1] = -4.0; w[2] = 6.0; w[3] = -4.0; w[4] = 1.0;
    return 2;
  }
  if (kind == 4 && order == 4) {
    w[0] = -1.0 / 6.0; w[1] = 2.0; w[2] = -13.0 / 2.0; w[3] = 28.0 / 3.0;
    w[4] = -13.0 / 2.0; w[5] = 2.0; w[6] = -1.0 / 6.0;
    return 3;
  }
  if (kind == 4 && order == 6) {
    w[0] = 7.0 / 240.0; w[1] = -2.0 / 5.0; w[2] = 169.0 / 60.0; w[3] = -122.0 / 15.0;
    w[4] = 91.0 / 8.0; w[5] = -122.0 / 15.0; w[6] = 169.0 / 60.0; w[7] = -2.0 / 5.0;
    w[8] = 7.0 / 240.0;
    return 4;
  }
  return -1;
}

/* ---- axis-extent precondition: diff/detail/PreconditionAxisExtent.hpp:64-79 */
static int require_axis(const char* axis, int N, int radius) {
  if (radius == 0) return 0;
  if (N == 1) return 0;
  if (N < 2 * radius + 1) {
    snprintf(g_err, sizeof g_err,
             "gridcalc: axis %s has N=%d but the requested stencil has radius %d, which requires "
             "N>=%d on a periodic grid (or N=1 for a degenerate axis)",
             axis, N, radius, 2 * radius + 1);
    return 1;
  }
  return 0;
}

static int require_axes(int nx, int ny, int nz, int r) {
  if (nx <= 0 || ny <= 0 || nz <= 0) {
    snprintf(g_err, sizeof g_err, "Grid: extents (Nx, Ny, Nz) must be > 0; got (%d, %d, %d)", nx, ny, nz);
    return 1;
  }
  if (require_axis("x", nx, r)) return 1;
  if (require_axis("y", ny, r)) return 1;
  if (require_axis("z", nz, r)) return 1;
  return 0;
}

#define MAXR 8

/* Wrapped index table: tab[i + MAXR] = ((i % N) + N) % N for i in [-MAXR, N+MAXR)
 * (core/IndexPolicy.hpp:28). */
static int* wrap_table(int N) {
  int* t = (int*)malloc(sizeof(int) * (size_t)(N + 2 * MAXR));
  for (int i = -MAXR; i < N + MAXR; ++i) t[i + MAXR] = ((i % N) + N) % N;
  return t;
}

typedef struct {
  int nx, ny, nz;
  int *wx, *wy, *wz;
} wrap3;

static void wrap3_init(wrap3* w, int nx, int ny, int nz) {
  w->nx = nx; w->ny = ny; w->nz = nz;
  w->wx = wrap_table(nx); w->wy = wrap_table(ny); w->wz = wrap_table(nz);
}
static void wrap3_free(wrap3* w) { free(w->wx); free(w->wy); free(w->wz); }

static inline size_t lin(const wrap3* w, int i, int j, int k) {
  return (size_t)w->wx[i + MAXR] +
         (size_t)w->nx * ((size_t)w->wy[j + MAXR] + (size_t)w->ny * (size_t)w->wz[k + MAXR]);
}

/* ---- diff/Laplacian.hpp:44-75 */
static void lap_core(const double* wt, int r, const wrap3* w, double ihx2, double ihy2, double ihz2,
                     const double* f, double* out) {
  for (int k = 0; k < w->nz; ++k)
    for (int j = 0; j < w->ny; ++j)
      for (int i = 0; i < w->nx; ++i) {
        double dxx = 0.0, dyy = 0.0, dzz = 0.0;
        for (int m = 0; m <= 2 * r; ++m) {
          const int off = m - r;
          dxx += wt[m] * f[lin(w, i + off, j, k)];
          dyy += wt[m] * f[lin(w, i, j + off, k)];
          dzz += wt[m] * f[lin(w, i, j, k + off)];
        }
        out[lin(w, i, j, k)] = dxx * ihx2 + dyy * ihy2 + dzz * ihz2;
      }
}

int oc_laplacian(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                 const double* in, double* out) {
  double wt[2 * MAXR + 1];
  const int r = oc_weights(2, order, wt);
  if (r < 0) { snprintf(g_err, sizeof g_err, "laplacian: unsupported order %d", order); return 1; }
  if (require_axes(nx, ny, nz, r)) return 1;
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  lap_core(wt, r, &w, 1.0 / (hx * hx), 1.0 / (hy * hy), 1.0 / (hz * hz), in, out);
  wrap3_free(&w);
  return 0;
}

/* ---- diff/detail/MultiIndexDerivative.hpp:96-137: d^(ax+ay+az) f / dx^ax dy^ay dz^az
   (the 31 named partials of diff/MixedPartial.hpp, ThirdOrder.hpp and
   FourthOrder.hpp forward here).  scale = 1 / h_a, divided once per
   derivative on each axis in x, y, z order; per point
   sum += (wx * (wy * wz)) * f over z taps, then y taps, then x taps, from
   0.0; result = sum * scale.  An axis with count 0 is the single tap 1.0. */
int oc_mixed(int ax, int ay, int az, int order, int nx, int ny, int nz, double hx, double hy, double hz,
             const double* f, double* out) {
  double wx[2 * MAXR + 1], wy[2 * MAXR + 1], wz[2 * MAXR + 1];
  int rx = 0, ry = 0, rz = 0;
  if (ax < 0 || ax > 4 || ay < 0 || ay > 4 || az < 0 || az > 4) {
    snprintf(g_err, sizeof g_err, "mixed: derivative counts must be in 0..4");
    return 1;
  }
  if (ax) rx = oc_weights(ax, order, wx); else wx[0] = 1.0;
  if (ay) ry = oc_weights(ay, order, wy); else wy[0] = 1.0;
  if (az) rz = oc_weights(az, order, wz); else wz[0] = 1.0;
  if (rx < 0 || ry < 0 || rz < 0) {
    snprintf(g_err, sizeof g_err, "mixed: unsupported order %d", order);
    return 1;
  }
  if (require_axis("x", nx, rx) || require_axis("y", ny, ry) || require_axis("z", nz, rz)) return 1;
  double scale = 1.0;
  for (int n = 0; n < ax; ++n) scale /= hx;
  for (int n = 0; n < ay; ++n) scale /= hy;
  for (int n = 0; n < az; ++n) scale /= hz;
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double sum = 0.0;
        for (int mz = 0; mz <= 2 * rz; ++mz)
          for (int my = 0; my <= 2 * ry; ++my) {
            const double wyz = wy[my] * wz[mz];
            for (int mx = 0; mx <= 2 * rx; ++mx)
              sum += wx[mx] * wyz * f[lin(&w, i + mx - rx, j + my - ry, k + mz - rz)];
          }
        out[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)] = sum * scale;
      }
  wrap3_free(&w);
  return 0;
}

/* ---- diff/Gradient.hpp:43-74 (scalar -> vector; output as three planes) */
int oc_gradient(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                const double* f, double* out3) {
  double wt[2 * MAXR + 1];
  const int r = oc_weights(1, order, wt);
  if (r < 0) { snprintf(g_err, sizeof g_err, "gradient: unsupported order %d", order); return 1; }
  if (require_axes(nx, ny, nz, r)) return 1;
  const double ihx = 1.0 / hx, ihy = 1.0 / hy, ihz = 1.0 / hz;
  const size_t n = (size_t)nx * ny * nz;
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double dx = 0.0, dy = 0.0, dz = 0.0;
        for (int m = 0; m <= 2 * r; ++m) {
          const int off = m - r;
          dx += wt[m] * f[lin(&w, i + off, j, k)];
          dy += wt[m] * f[lin(&w, i, j + off, k)];
          dz += wt[m] * f[lin(&w, i, j, k + off)];
        }
        const size_t c = lin(&w, i, j, k);
        out3[c] = dx * ihx;
        out3[n + c] = dy * ihy;
        out3[2 * n + c] = dz * ihz;
      }
  wrap3_free(&w);
  return 0;
}

/* ---- diff/Divergence.hpp:43-74 (vector as three planes -> scalar) */
int oc_divergence(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                  const double* v3, double* out) {
  double wt[2 * MAXR + 1];
  const int r = oc_weights(1, order, wt);
  if (r < 0) { snprintf(g_err, sizeof g_err, "divergence: unsupported order %d", order); return 1; }
  if (require_axes(nx, ny, nz, r)) return 1;
  const double ihx = 1.0 / hx, ihy = 1.0 / hy, ihz = 1.0 / hz;
  const size_t n = (size_t)nx * ny * nz;
  const double *vx = v3, *vy = v3 + n, *vz = v3 + 2 * n;
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int m = 0; m <= 2 * r; ++m) {
          const int off = m - r;
          a += wt[m] * vx[lin(&w, i + off, j, k)];
          b += wt[m] * vy[lin(&w, i, j + off, k)];
          c += wt[m] * vz[lin(&w, i, j, k + off)];
        }
        out[lin(&w, i, j, k)] = a * ihx + b * ihy + c * ihz;
      }
  wrap3_free(&w);
  return 0;
}

/* ---- diff/Gradient.hpp:100-137 (rank-2: Vec3d -> Mat3d).  Row `comp` of
 * M = grad v is the scalar gradient of component `comp`, with the same taps,
 * zero-initialised sums and 1/h scaling, so each row is one scalar pass.
 * Layout: three input planes (x, y, z); nine output planes, plane
 * 3*comp + axis holding M(comp, axis) = d_axis v_comp. */
int oc_gradient_vec(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                    const double* v3, double* out9) {
  const size_t n = (size_t)nx * ny * nz;
  for (int comp = 0; comp < 3; ++comp)
    if (oc_gradient(order, nx, ny, nz, hx, hy, hz, v3 + comp * n, out9 + 3 * comp * n)) return 1;
  return 0;
}

/* ---- diff/Divergence.hpp:100-135 (rank-lowering: Mat3d -> Vec3d).
 * (div M)_comp = d_x M(comp,0) + d_y M(comp,1) + d_z M(comp,2), summed as
 * (dx/hx + dy/hy) + dz/hz exactly like the vector divergence, so component
 * `comp` is the vector divergence of row `comp` (planes 3*comp .. 3*comp+2). */
int oc_divergence_mat(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                      const double* m9, double* out3) {
  const size_t n = (size_t)nx * ny * nz;
  for (int comp = 0; comp < 3; ++comp)
    if (oc_divergence(order, nx, ny, nz, hx, hy, hz, m9 + 3 * comp * n, out3 + comp * n)) return 1;
  return 0;
}

/* ---- diff/Biharmonic.hpp:48-104 */
int oc_biharmonic(int order, int nx, int ny, int nz, double hx, double hy, double hz,
                  const double* f, double* out) {
  double w2[2 * MAXR + 1], w4[2 * MAXR + 1];
  const int r2 = oc_weights(2, order, w2);
  const int r4 = oc_weights(4, order, w4);
  if (r2 < 0 || r4 < 0) { snprintf(g_err, sizeof g_err, "biharmonic: unsupported order %d", order); return 1; }
  const int rmax = r4 > r2 ? r4 : r2;
  if (require_axes(nx, ny, nz, rmax)) return 1;
  const double ihx2 = 1.0 / (hx * hx), ihy2 = 1.0 / (hy * hy), ihz2 = 1.0 / (hz * hz);
  const double ihx4 = ihx2 * ihx2, ihy4 = ihy2 * ihy2, ihz4 = ihz2 * ihz2;
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double dx4 = 0.0, dy4 = 0.0, dz4 = 0.0;
        for (int m = 0; m <= 2 * r4; ++m) {
          const int off = m - r4;
          dx4 += w4[m] * f[lin(&w, i + off, j, k)];
          dy4 += w4[m] * f[lin(&w, i, j + off, k)];
          dz4 += w4[m] * f[lin(&w, i, j, k + off)];
        }
        double dx2y2 = 0.0, dx2z2 = 0.0, dy2z2 = 0.0;
        for (int mb = 0; mb <= 2 * r2; ++mb) {
          const int ob = mb - r2;
          const double wb = w2[mb];
          for (int ma = 0; ma <= 2 * r2; ++ma) {
            const int oa = ma - r2;
            const double wab = w2[ma] * wb;
            dx2y2 += wab * f[lin(&w, i + oa, j + ob, k)];
            dx2z2 += wab * f[lin(&w, i + oa, j, k + ob)];
            dy2z2 += wab * f[lin(&w, i, j + oa, k + ob)];
          }
        }
        out[lin(&w, i, j, k)] = dx4 * ihx4 + dy4 * ihy4 + dz4 * ihz4 +
                                2.0 * (dx2y2 * ihx2 * ihy2 + dx2z2 * ihx2 * ihz2 + dy2z2 * ihy2 * ihz2);
      }
  wrap3_free(&w);
  return 0;
}

/* ---- fvm/CellLaplacian.hpp:48-50 */
static inline double hmean(double a, double b) { return 2.0 * a * b / (a + b); }

/* ---- fvm/CellLaplacian.hpp:91-143 */
int oc_cell_laplacian(int nx, int ny, int nz, double hx, double hy, double hz,
                      const double* psi, const double* D, double* out, int64_t* bad_index) {
  if (require_axes(nx, ny, nz, 1)) return 1;
  const size_t n = (size_t)nx * ny * nz;
  for (size_t idx = 0; idx < n; ++idx) {
    if (!(D[idx] > 0.0)) {
      if (bad_index) *bad_index = (int64_t)idx;
      snprintf(g_err, sizeof g_err,
               "fvm::cellLaplacian: D must be strictly positive at every cell; first violation "
               "at flat index %lld with D=%f", (long long)idx, D[idx]);
      return 2;
    }
  }
  const double ihx2 = 1.0 / (hx * hx), ihy2 = 1.0 / (hy * hy), ihz2 = 1.0 / (hz * hz);
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const size_t c = lin(&w, i, j, k);
        const double pc = psi[c], Dc = D[c];
        const double Dxp = hmean(Dc, D[lin(&w, i + 1, j, k)]);
        const double Dxm = hmean(D[lin(&w, i - 1, j, k)], Dc);
        const double Dyp = hmean(Dc, D[lin(&w, i, j + 1, k)]);
        const double Dym = hmean(D[lin(&w, i, j - 1, k)], Dc);
        const double Dzp = hmean(Dc, D[lin(&w, i, j, k + 1)]);
        const double Dzm = hmean(D[lin(&w, i, j, k - 1)], Dc);
        const double rx = (Dxp * (psi[lin(&w, i + 1, j, k)] - pc) - Dxm * (pc - psi[lin(&w, i - 1, j, k)])) * ihx2;
        const double ry = (Dyp * (psi[lin(&w, i, j + 1, k)] - pc) - Dym * (pc - psi[lin(&w, i, j - 1, k)])) * ihy2;
        const double rz = (Dzp * (psi[lin(&w, i, j, k + 1)] - pc) - Dzm * (pc - psi[lin(&w, i, j, k - 1)])) * ihz2;
        out[c] = rx + ry + rz;
      }
  wrap3_free(&w);
  return 0;
}

/* ---- func/Integrate.hpp:65-74 (recursive pairwise, base case 64) */
double oc_sum_pairwise(const double* x, size_t n) {
  if (n <= 64) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += x[i];
    return s;
  }
  const size_t mid = n / 2;
  return oc_sum_pairwise(x, mid) + oc_sum_pairwise(x + mid, n - mid);
}

/* ---- func/Integrate.hpp:85-99 (Neumaier) */
double oc_sum_neumaier(const double* x, size_t n) {
  double sum = 0.0, c = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const double v = x[i];
    const double t = sum + v;
    if (fabs(sum) >= fabs(v)) c += (sum - t) + v;
    else c += (v - t) + sum;
    sum = t;
  }
  return sum + c;
}

/* ---- func/Integrate.hpp:116-135 */
double oc_integrate(int nx, int ny, int nz, double hx, double hy, double hz, const double* in,
                    int kahan) {
  const size_t n = (size_t)nx * ny * nz;
  const double vol = hx * hy * hz;
  return vol * (kahan ? oc_sum_neumaier(in, n) : oc_sum_pairwise(in, n));
}

/* ---- examples/common/cahn_hilliard.hpp:38-59 at a selectable Laplacian order */
static void ch_rhs_core(const double* wt, int r, const wrap3* w, double ihx2, double ihy2,
                        double ihz2, double M, double kappa, const double* psi, double* lap,
                        double* mu, double* out) {
  const size_t n = (size_t)w->nx * w->ny * w->nz;
  lap_core(wt, r, w, ihx2, ihy2, ihz2, psi, lap);
  for (size_t idx = 0; idx < n; ++idx) {
    const double p = psi[idx];
    mu[idx] = -p + p * p * p - kappa * lap[idx];
  }
  lap_core(wt, r, w, ihx2, ihy2, ihz2, mu, out);
  for (size_t idx = 0; idx < n; ++idx) out[idx] *= M;
}

int oc_ch_rhs(int order, double M, double kappa, int nx, int ny, int nz, double hx, double hy,
              double hz, const double* psi, double* out) {
  double wt[2 * MAXR + 1];
  const int r = oc_weights(2, order, wt);
  if (r < 0) { snprintf(g_err, sizeof g_err, "ch: unsupported order %d", order); return 1; }
  if (require_axes(nx, ny, nz, r)) return 1;
  const size_t n = (size_t)nx * ny * nz;
  double* lap = (double*)malloc(sizeof(double) * n);
  double* mu = (double*)malloc(sizeof(double) * n);
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  ch_rhs_core(wt, r, &w, 1.0 / (hx * hx), 1.0 / (hy * hy), 1.0 / (hz * hz), M, kappa, psi, lap, mu, out);
  wrap3_free(&w);
  free(lap); free(mu);
  return 0;
}

/* RHS kinds driven by the integrators below. */
typedef struct {
  int kind; /* 0 = CH, 1 = constant-D Laplacian (order 2), 2 = FVM cell Laplacian */
  const double* wt; int r;
  const wrap3* w;
  double ihx2, ihy2, ihz2, M, kappa;
  const double* D;
  double *lap, *mu;
} rhs_ctx;

static void rhs_eval(const rhs_ctx* c, const double* psi, double* out) {
  if (c->kind == 0) {
    ch_rhs_core(c->wt, c->r, c->w, c->ihx2, c->ihy2, c->ihz2, c->M, c->kappa, psi, c->lap, c->mu, out);
  } else if (c->kind == 1) {
    lap_core(c->wt, c->r, c->w, c->ihx2, c->ihy2, c->ihz2, psi, out);
  } else {
    const wrap3* w = c->w;
    for (int k = 0; k < w->nz; ++k)
      for (int j = 0; j < w->ny; ++j)
        for (int i = 0; i < w->nx; ++i) {
          const double* D = c->D;
          const size_t q = lin(w, i, j, k);
          const double pc = psi[q], Dc = D[q];
          const double Dxp = hmean(Dc, D[lin(w, i + 1, j, k)]);
          const double Dxm = hmean(D[lin(w, i - 1, j, k)], Dc);
          const double Dyp = hmean(Dc, D[lin(w, i, j + 1, k)]);
          const double Dym = hmean(D[lin(w, i, j - 1, k)], Dc);
          const double Dzp = hmean(Dc, D[lin(w, i, j, k + 1)]);
          const double Dzm = hmean(D[lin(w, i, j, k - 1)], Dc);
          const double rx = (Dxp * (psi[lin(w, i + 1, j, k)] - pc) - Dxm * (pc - psi[lin(w, i - 1, j, k)])) * c->ihx2;
          const double ry = (Dyp * (psi[lin(w, i, j + 1, k)] - pc) - Dym * (pc - psi[lin(w, i, j - 1, k)])) * c->ihy2;
          const double rz = (Dzp * (psi[lin(w, i, j, k + 1)] - pc) - Dzm * (pc - psi[lin(w, i, j, k - 1)])) * c->ihz2;
          out[q] = rx + ry + rz;
        }
  }
}

/* ---- solve/RK4.hpp:99-154 and solve/ExplicitEuler.hpp:79-112 */
static void time_integrate(const rhs_ctx* c, double* psi, size_t n, double dt, int n_steps,
                           int integrator) {
  if (integrator == 0) {
    double* tmp = (double*)malloc(sizeof(double) * n);
    for (int s = 0; s < n_steps; ++s) {
      rhs_eval(c, psi, tmp);
      for (size_t q = 0; q < n; ++q) psi[q] += dt * tmp[q];
    }
    free(tmp);
    return;
  }
  double* k1 = (double*)malloc(sizeof(double) * n);
  double* k2 = (double*)malloc(sizeof(double) * n);
  double* k3 = (double*)malloc(sizeof(double) * n);
  double* k4 = (double*)malloc(sizeof(double) * n);
  double* y = (double*)malloc(sizeof(double) * n);
  const double half_dt = 0.5 * dt, sixth_dt = dt / 6.0, third_dt = dt / 3.0;
  for (int s = 0; s < n_steps; ++s) {
    rhs_eval(c, psi, k1);
    for (size_t q = 0; q < n; ++q) y[q] = psi[q] + half_dt * k1[q];
    rhs_eval(c, y, k2);
    for (size_t q = 0; q < n; ++q) y[q] = psi[q] + half_dt * k2[q];
    rhs_eval(c, y, k3);
    for (size_t q = 0; q < n; ++q) y[q] = psi[q] + dt * k3[q];
    rhs_eval(c, y, k4);
    for (size_t q = 0; q < n; ++q) psi[q] += sixth_dt * (k1[q] + k4[q]) + third_dt * (k2[q] + k3[q]);
  }
  free(k1); free(k2); free(k3); free(k4); free(y);
}

static int check_steps(const char* who, double dt, int n_steps) {
  if (n_steps < 0) { snprintf(g_err, sizeof g_err, "%s: n_steps must be >= 0; got %d", who, n_steps); return 1; }
  if (dt < 0.0) { snprintf(g_err, sizeof g_err, "%s: dt must be >= 0; got %f", who, dt); return 1; }
  return 0;
}

int oc_ch_integrate(int order, double M, double kappa, int nx, int ny, int nz, double hx,
                    double hy, double hz, double* psi, double dt, int n_steps, int integrator) {
  double wt[2 * MAXR + 1];
  const int r = oc_weights(2, order, wt);
  if (r < 0) { snprintf(g_err, sizeof g_err, "ch: unsupported order %d", order); return 1; }
  if (check_steps("solve::integrate", dt, n_steps)) return 1;
  /* the reference reaches the axis check only through the first RHS call */
  if (n_steps > 0 && require_axes(nx, ny, nz, r)) return 1;
  const size_t n = (size_t)nx * ny * nz;
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  rhs_ctx c = {0, wt, r, &w, 1.0 / (hx * hx), 1.0 / (hy * hy), 1.0 / (hz * hz), M, kappa, NULL,
               (double*)malloc(sizeof(double) * n), (double*)malloc(sizeof(double) * n)};
  time_integrate(&c, psi, n, dt, n_steps, integrator);
  free(c.lap); free(c.mu);
  wrap3_free(&w);
  return 0;
}

/* ---- func/Functional.hpp:88-148 (two-argument form) over
 * examples/common/cahn_hilliard.hpp:64-77: integrand from the order-2
 * gradient, summed pairwise. mode 0 = free energy, 1 = |grad psi|^2. */
static double ch_energy(int mode, int nx, int ny, int nz, double hx, double hy, double hz,
                        const double* psi, double kappa) {
  const size_t n = (size_t)nx * ny * nz;
  double* g = (double*)malloc(sizeof(double) * 3 * n);
  double* f = (double*)malloc(sizeof(double) * n);
  oc_gradient(2, nx, ny, nz, hx, hy, hz, psi, g);
  for (size_t q = 0; q < n; ++q) {
    const double gx = g[q], gy = g[n + q], gz = g[2 * n + q];
    const double sq = gx * gx + gy * gy + gz * gz;
    const double p = psi[q];
    f[q] = mode == 0 ? -0.5 * p * p + 0.25 * p * p * p * p + 0.5 * kappa * sq : sq;
  }
  const double r = (hx * hy * hz) * oc_sum_pairwise(f, n);
  free(g); free(f);
  return r;
}

double oc_ch_free_energy(int nx, int ny, int nz, double hx, double hy, double hz,
                         const double* psi, double kappa) {
  return ch_energy(0, nx, ny, nz, hx, hy, hz, psi, kappa);
}

double oc_ch_gradient_energy(int nx, int ny, int nz, double hx, double hy, double hz,
                             const double* psi) {
  return ch_energy(1, nx, ny, nz, hx, hy, hz, psi, 0.0);
}

/* ---- examples/common/cahn_hilliard.hpp:108-113 */
double oc_ch_mean(int nx, int ny, int nz, double hx, double hy, double hz, const double* psi) {
  const size_t n = (size_t)nx * ny * nz;
  const double vol = hx * hy * hz;
  const double total = (double)n * vol;
  return vol * oc_sum_pairwise(psi, n) / total;
}

/* ---- solve/Diffusion.hpp:187-207 */
double oc_d_max_face(int nx, int ny, int nz, const double* D) {
  double m = 0.0;
  for (int k = 0; k < nz; ++k) {
    const int kp = (k + 1) % nz;
    for (int j = 0; j < ny; ++j) {
      const int jp = (j + 1) % ny;
      for (int i = 0; i < nx; ++i) {
        const int ip = (i + 1) % nx;
        const double Dc = D[i + (size_t)nx * (j + (size_t)ny * k)];
        const double fx = hmean(Dc, D[ip + (size_t)nx * (j + (size_t)ny * k)]);
        const double fy = hmean(Dc, D[i + (size_t)nx * (jp + (size_t)ny * k)]);
        const double fz = hmean(Dc, D[i + (size_t)nx * (j + (size_t)ny * kp)]);
        if (fx > m) m = fx;
        if (fy > m) m = fy;
        if (fz > m) m = fz;
      }
    }
  }
  return m;
}

/* ---- solve/Diffusion.hpp:45-59 */
static int check_cfl(double limit, double hx, double hy, double hz, double D, double dt) {
  const double inv_sum = 1.0 / (hx * hx) + 1.0 / (hy * hy) + 1.0 / (hz * hz);
  const double cfl = D * dt * inv_sum;
  if (cfl > limit) {
    snprintf(g_err, sizeof g_err,
             "solve::diffuse: explicit-diffusion CFL violated: D*dt*(1/hx^2 + 1/hy^2 + 1/hz^2) = %f > %f",
             cfl, limit);
    return 1;
  }
  return 0;
}

/* ---- solve/Diffusion.hpp:89-112 */
int oc_diffuse_const(int nx, int ny, int nz, double hx, double hy, double hz, double* psi,
                     double D, double dt, int n_steps, int integrator) {
  if (D < 0.0) { snprintf(g_err, sizeof g_err, "solve::diffuse: D must be >= 0; got %f", D); return 1; }
  if (dt < 0.0) { snprintf(g_err, sizeof g_err, "solve::diffuse: dt must be >= 0; got %f", dt); return 1; }
  if (n_steps < 0) { snprintf(g_err, sizeof g_err, "solve::diffuse: n_steps must be >= 0; got %d", n_steps); return 1; }
  if (check_cfl(integrator ? 0.6963 : 0.5, hx, hy, hz, D, dt)) return 1;
  double wt[3];
  const int r = oc_weights(2, 2, wt);
  if (n_steps > 0 && require_axes(nx, ny, nz, r)) return 1;
  const size_t n = (size_t)nx * ny * nz;
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  rhs_ctx c = {1, wt, r, &w, 1.0 / (hx * hx), 1.0 / (hy * hy), 1.0 / (hz * hz), 0, 0, NULL, NULL, NULL};
  time_integrate(&c, psi, n, D * dt, n_steps, integrator);
  wrap3_free(&w);
  return 0;
}

/* ---- solve/Diffusion.hpp:161-216 */
int oc_diffuse_fvm(int nx, int ny, int nz, double hx, double hy, double hz, double* psi,
                   const double* D, double dt, int n_steps, int integrator) {
  if (dt < 0.0) { snprintf(g_err, sizeof g_err, "solve::diffuse: dt must be >= 0; got %f", dt); return 1; }
  if (n_steps < 0) { snprintf(g_err, sizeof g_err, "solve::diffuse: n_steps must be >= 0; got %d", n_steps); return 1; }
  const double dmax = oc_d_max_face(nx, ny, nz, D);
  if (check_cfl(integrator ? 0.6963 : 0.5, hx, hy, hz, dmax, dt)) return 1;
  /* the reference reaches these checks only through the first RHS call
   * (fvm/CellLaplacian.hpp:95-109) */
  if (n_steps > 0 && require_axes(nx, ny, nz, 1)) return 1;
  const size_t n = (size_t)nx * ny * nz;
  for (size_t q = 0; n_steps > 0 && q < n; ++q)
    if (!(D[q] > 0.0)) {
      snprintf(g_err, sizeof g_err,
               "fvm::cellLaplacian: D must be strictly positive at every cell; first violation "
               "at flat index %zu", q);
      return 2;
    }
  wrap3 w; wrap3_init(&w, nx, ny, nz);
  rhs_ctx c = {2, NULL, 1, &w, 1.0 / (hx * hx), 1.0 / (hy * hy), 1.0 / (hz * hz), 0, 0, D, NULL, NULL};
  time_integrate(&c, psi, n, dt, n_steps, integrator);
  wrap3_free(&w);
  return 0;
}

/* ---- func/Functional.hpp:88-148 (scalar) and :183-220 (vector): evaluate a
 * callable per cell into an integrand field, then func::integrate.  The
 * derivative fields of the callable's arity are materialised first, at the
 * reference's default order 2 and in its order (gradient, Laplacian,
 * biharmonic), so the first failing extent check is the reference's. */
static double oc_run_program(const oc_instr* prog, int n_instr, const double* in) {
  double r[32];
  for (int pc = 0; pc < n_instr; ++pc) {
    const oc_instr* I = &prog[pc];
    double v;
    switch (I->op) {
      case 0: v = I->value; break;
      case 1: v = in[I->a]; break;
      case 2: v = r[I->a] + r[I->b]; break;
      case 3: v = r[I->a] - r[I->b]; break;
      case 4: v = r[I->a] * r[I->b]; break;
      case 5: v = r[I->a] / r[I->b]; break;
      case 6: v = -r[I->a]; break;
      case 7: v = fabs(r[I->a]); break;
      case 8: v = sqrt(r[I->a]); break;
      case 9: v = r[I->b] < r[I->a] ? r[I->b] : r[I->a]; break;
      default: v = r[I->a] < r[I->b] ? r[I->b] : r[I->a]; break;
    }
    r[I->dst] = v;
  }
  return r[prog[n_instr - 1].dst];
}

int oc_evaluate_program(int components, int arity, int nx, int ny, int nz, double hx, double hy, double hz,
                        const double* field, const oc_instr* prog, int n_instr, int kahan, double* result) {
  if (!((components == 1 && arity >= 1 && arity <= 4) || (components == 3 && arity >= 1 && arity <= 2)) ||
      n_instr < 1 || n_instr > 128) {
    snprintf(g_err, sizeof g_err, "evaluate: bad program shape");
    return 3;
  }
  for (int pc = 0; pc < n_instr; ++pc)
    if (prog[pc].op < 0 || prog[pc].op > 10 || prog[pc].dst < 0 || prog[pc].dst >= 32 || prog[pc].a < 0 ||
        prog[pc].a >= 32 || prog[pc].b < 0 || prog[pc].b >= 32) {
      snprintf(g_err, sizeof g_err, "evaluate: bad instruction %d", pc);
      return 3;
    }
  const size_t n = (size_t)nx * ny * nz;
  const int nin = components == 1 ? (arity == 1 ? 1 : arity + 2) : (arity == 1 ? 3 : 12);
  for (int pc = 0; pc < n_instr; ++pc)
    if (prog[pc].op == 1 && prog[pc].a >= nin) {
      snprintf(g_err, sizeof g_err, "evaluate: input %d beyond the arity", prog[pc].a);
      return 3;
    }
  double* d1 = NULL; double* d2 = NULL; double* d4 = NULL;
  double* integrand = (double*)malloc(sizeof(double) * (n ? n : 1));
  int rc = 0;
  if (components == 1) {
    if (arity >= 2) { d1 = (double*)malloc(sizeof(double) * 3 * n); rc = oc_gradient(2, nx, ny, nz, hx, hy, hz, field, d1); }
    if (!rc && arity >= 3) { d2 = (double*)malloc(sizeof(double) * n); rc = oc_laplacian(2, nx, ny, nz, hx, hy, hz, field, d2); }
    if (!rc && arity >= 4) { d4 = (double*)malloc(sizeof(double) * n); rc = oc_biharmonic(2, nx, ny, nz, hx, hy, hz, field, d4); }
  } else if (arity >= 2) {
    d1 = (double*)malloc(sizeof(double) * 9 * n);
    rc = oc_gradient_vec(2, nx, ny, nz, hx, hy, hz, field, d1);
  }
  if (!rc) {
    for (size_t c = 0; c < n; ++c) {
      double in[12];
      if (components == 1) {
        in[0] = field[c];
        if (arity >= 2) { in[1] = d1[c]; in[2] = d1[n + c]; in[3] = d1[2 * n + c]; }
        if (arity >= 3) in[4] = d2[c];
        if (arity >= 4) in[5] = d4[c];
      } else {
        for (int q = 0; q < 3; ++q) in[q] = field[q * n + c];
        if (arity >= 2) for (int q = 0; q < 9; ++q) in[3 + q] = d1[q * n + c];
      }
      integrand[c] = oc_run_program(prog, n_instr, in);
    }
    if (!rc) *result = oc_integrate(nx, ny, nz, hx, hy, hz, integrand, kahan);
  }
  free(d1); free(d2); free(d4); free(integrand);
  return rc;
}
