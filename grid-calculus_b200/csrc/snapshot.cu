// Snapshot output and checkpoint / resume.
//
// * VTK: the reference's legacy STRUCTURED_POINTS writer
//   (examples/common/vtk_writer.hpp:34-66) reproduced byte for byte in its
//   ASCII form (17 significant digits, i fastest), plus a BINARY form of the
//   same header with big-endian doubles.
// * Checkpoints: a fixed little-endian header (magic, version, dtype, grid,
//   components, sizes, a 64-bit checksum of the whole file), a JSON metadata
//   string, then the raw field planes.  Loading one and continuing a
//   trajectory gives the bit-identical state of an uninterrupted run.
// * gc_snapshotter: snapshots of device fields that do not stall the
//   computation.  The field is first copied device-to-device on the
//   context's stream into one of `depth` device slots (at HBM speed, so the
//   next step may overwrite the field right away); a copy stream then moves
//   the slot to pinned host memory over PCIe while later steps run, and a
//   writer thread formats and writes the file once that copy completes.  A
//   slot is reused only after its file is written.
#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace gcb {
namespace {

constexpr char kCkptMagic[8] = {'G', 'C', 'B', '2', '0', '0', 'C', 'K'};
// Version 2: the checksum covers the header, the metadata and the data.
// Version 1 files (checksum of the data only) are still read.
constexpr uint32_t kCkptVersion = 2;

struct CkptHeader {
  char magic[8];
  uint32_t version;
  uint32_t dtype;
  int32_t nx, ny, nz, components;
  double hx, hy, hz;
  uint64_t data_bytes;
  uint64_t meta_len;
  uint64_t checksum;
};
static_assert(sizeof(CkptHeader) == 80, "checkpoint header layout");

// 64-bit checksum of a byte string: a multiply-rotate mix over 8-byte
// little-endian words (the last one zero-padded), seeded with the length.
uint64_t checksum64(const void* data, uint64_t bytes) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  uint64_t h = 0x9E3779B97F4A7C15ull ^ bytes;
  uint64_t i = 0;
  for (; i + 8 <= bytes; i += 8) {
    uint64_t w;
    std::memcpy(&w, p + i, 8);
    h ^= w * 0xFF51AFD7ED558CCDull;
    h = ((h << 27) | (h >> 37)) * 0x9E3779B97F4A7C15ull + 0x52DCE729ull;
  }
  if (i < bytes) {
    uint64_t w = 0;
    std::memcpy(&w, p + i, static_cast<size_t>(bytes - i));
    h ^= w * 0xFF51AFD7ED558CCDull;
    h = ((h << 27) | (h >> 37)) * 0x9E3779B97F4A7C15ull + 0x52DCE729ull;
  }
  h ^= h >> 33;
  h *= 0xC4CEB9FE1A85EC53ull;
  return h ^ (h >> 29);
}

// Checksum of a version-2 file: the header with its checksum field zero,
// the metadata and the data are each hashed and the three hashes hashed
// together, so a changed bit anywhere in the file fails the check (every
// step of checksum64 is a bijection of its state for a given length).
uint64_t file_checksum(const CkptHeader& h, const std::string& meta, const void* data) {
  CkptHeader z = h;
  z.checksum = 0;
  const uint64_t parts[3] = {checksum64(&z, sizeof z), checksum64(meta.data(), meta.size()),
                             checksum64(data, h.data_bytes)};
  return checksum64(parts, sizeof parts);
}

std::string g17(double v) {
  char buf[40];
  std::snprintf(buf, sizeof buf, "%.17g", v);
  return buf;
}

inline double value_at(const void* host, gc_dtype dt, size_t i) {
  return dt == GC_F64 ? static_cast<const double*>(host)[i] : static_cast<double>(static_cast<const float*>(host)[i]);
}

gc_status write_vtk_file(const gc_grid* g, gc_dtype dt, const void* host, const std::string& path,
                         const std::string& name, gc_vtk_encoding enc) {
  std::FILE* out = std::fopen(path.c_str(), "wb");
  if (!out) return fail(GC_ERR_IO, "writeVtkStructuredPoints: cannot open '" + path + "' for writing");
  const size_t n = cells(g);
  std::string head = "# vtk DataFile Version 3.0\n";
  head += "gridcalc field: " + name + "\n";
  head += enc == GC_VTK_BINARY ? "BINARY\n" : "ASCII\n";
  head += "DATASET STRUCTURED_POINTS\n";
  head += "DIMENSIONS " + std::to_string(g->nx) + ' ' + std::to_string(g->ny) + ' ' + std::to_string(g->nz) + '\n';
  head += "ORIGIN 0 0 0\n";
  head += "SPACING " + g17(g->hx) + ' ' + g17(g->hy) + ' ' + g17(g->hz) + '\n';
  head += "POINT_DATA " + std::to_string(n) + '\n';
  head += "SCALARS " + name + " double 1\n";
  head += "LOOKUP_TABLE default\n";
  bool ok = std::fwrite(head.data(), 1, head.size(), out) == head.size();
  if (enc == GC_VTK_BINARY) {
    std::vector<unsigned char> buf;
    const size_t block = 1 << 20;
    for (size_t b = 0; ok && b < n; b += block) {
      const size_t m = std::min(block, n - b);
      buf.resize(8 * m);
      for (size_t i = 0; i < m; ++i) {
        const double v = value_at(host, dt, b + i);
        uint64_t w;
        std::memcpy(&w, &v, 8);
        for (int q = 0; q < 8; ++q) buf[8 * i + q] = static_cast<unsigned char>(w >> (56 - 8 * q));
      }
      ok = std::fwrite(buf.data(), 1, buf.size(), out) == buf.size();
    }
    ok = ok && std::fputc('\n', out) != EOF;
  } else {
    // Values are formatted in parallel blocks (the format is %.17g, one
    // value per line) and written in order.
    const size_t block = 1 << 16;
    const size_t nblocks = (n + block - 1) / block;
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t batch = static_cast<size_t>(hw) * 4;
    std::vector<std::string> text(batch);
    for (size_t b0 = 0; ok && b0 < nblocks; b0 += batch) {
      const size_t nb = std::min(batch, nblocks - b0);
      auto format = [&](size_t t) {
        for (size_t q = t; q < nb; q += hw) {
          const size_t lo = (b0 + q) * block, hi = std::min(n, lo + block);
          std::string& s = text[q];
          s.clear();
          s.reserve((hi - lo) * 25);
          char buf[40];
          for (size_t i = lo; i < hi; ++i) {
            const int len = std::snprintf(buf, sizeof buf, "%.17g\n", value_at(host, dt, i));
            s.append(buf, static_cast<size_t>(len));
          }
        }
      };
      std::vector<std::thread> pool;
      for (unsigned t = 1; t < hw && t < nb; ++t) pool.emplace_back(format, t);
      format(0);
      for (auto& th : pool) th.join();
      for (size_t q = 0; ok && q < nb; ++q) ok = std::fwrite(text[q].data(), 1, text[q].size(), out) == text[q].size();
    }
  }
  ok = (std::fclose(out) == 0) && ok;
  if (!ok) return fail(GC_ERR_IO, "writeVtkStructuredPoints: write to '" + path + "' failed");
  return GC_OK;
}

gc_status write_ckpt_file(const gc_grid* g, gc_dtype dt, int comps, const void* host, const std::string& path,
                          const std::string& meta) {
  CkptHeader h{};
  std::memcpy(h.magic, kCkptMagic, 8);
  h.version = kCkptVersion;
  h.dtype = static_cast<uint32_t>(dt);
  h.nx = g->nx; h.ny = g->ny; h.nz = g->nz; h.components = comps;
  h.hx = g->hx; h.hy = g->hy; h.hz = g->hz;
  h.data_bytes = static_cast<uint64_t>(cells(g)) * comps * dtype_size(dt);
  h.meta_len = meta.size();
  h.checksum = file_checksum(h, meta, host);
  // Written to a temporary name and renamed, so a crash never leaves a
  // truncated file under the final name.
  const std::string tmp = path + ".part";
  std::FILE* out = std::fopen(tmp.c_str(), "wb");
  if (!out) return fail(GC_ERR_IO, "checkpoint: cannot open '" + tmp + "' for writing");
  bool ok = std::fwrite(&h, sizeof h, 1, out) == 1;
  ok = ok && (meta.empty() || std::fwrite(meta.data(), 1, meta.size(), out) == meta.size());
  ok = ok && (h.data_bytes == 0 || std::fwrite(host, 1, h.data_bytes, out) == h.data_bytes);
  ok = (std::fclose(out) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
    std::remove(tmp.c_str());
    return fail(GC_ERR_IO, "checkpoint: write to '" + path + "' failed");
  }
  return GC_OK;
}

gc_status read_ckpt_header(std::FILE* in, const std::string& path, CkptHeader* h) {
  if (std::fread(h, sizeof *h, 1, in) != 1 || std::memcmp(h->magic, kCkptMagic, 8) != 0)
    return fail(GC_ERR_IO, "checkpoint: '" + path + "' is not a gridcalc_b200 checkpoint");
  if (h->version != 1 && h->version != kCkptVersion)
    return fail(GC_ERR_UNSUPPORTED, "checkpoint: '" + path + "' has version " + std::to_string(h->version));
  if ((h->dtype != GC_F64 && h->dtype != GC_F32) || h->nx <= 0 || h->ny <= 0 || h->nz <= 0 || h->components <= 0 ||
      h->data_bytes != static_cast<uint64_t>(h->nx) * h->ny * h->nz * h->components * (h->dtype == GC_F64 ? 8 : 4))
    return fail(GC_ERR_IO, "checkpoint: '" + path + "' has an inconsistent header");
  // The sizes must add up to the file's, before anyone sizes a buffer by them.
  const off_t at = ftello(in);
  if (at < 0 || fseeko(in, 0, SEEK_END) != 0) return fail(GC_ERR_IO, "checkpoint: cannot read '" + path + "'");
  const off_t end = ftello(in);
  if (end < 0 || fseeko(in, at, SEEK_SET) != 0) return fail(GC_ERR_IO, "checkpoint: cannot read '" + path + "'");
  const uint64_t size = static_cast<uint64_t>(end), body = size - sizeof *h;
  if (h->meta_len > body || h->data_bytes > body - h->meta_len)
    return fail(GC_ERR_IO, "checkpoint: '" + path + "' is truncated");
  if (h->meta_len + h->data_bytes != body)
    return fail(GC_ERR_IO, "checkpoint: '" + path + "' has an inconsistent header");
  return GC_OK;
}

gc_status read_ckpt(const std::string& path, CkptHeader* h, std::string* meta, void* host, size_t host_bytes) {
  std::FILE* in = std::fopen(path.c_str(), "rb");
  if (!in) return fail(GC_ERR_IO, "checkpoint: cannot open '" + path + "'");
  gc_status s = read_ckpt_header(in, path, h);
  // The metadata is read whenever the data is (a version-2 checksum covers it).
  std::string local;
  std::string* m = meta ? meta : (host ? &local : nullptr);
  if (s == GC_OK && m) {
    m->assign(static_cast<size_t>(h->meta_len), '\0');
    if (h->meta_len && std::fread(&(*m)[0], 1, static_cast<size_t>(h->meta_len), in) != h->meta_len)
      s = fail(GC_ERR_IO, "checkpoint: '" + path + "' is truncated");
  }
  if (s == GC_OK && host) {
    if (host_bytes < h->data_bytes) {
      s = fail(GC_ERR_INVALID_ARG, "checkpoint: buffer of " + std::to_string(host_bytes) + " bytes, field has " +
                                       std::to_string(h->data_bytes));
    } else if (h->data_bytes && std::fread(host, 1, h->data_bytes, in) != h->data_bytes) {
      s = fail(GC_ERR_IO, "checkpoint: '" + path + "' is truncated");
    } else if ((h->version == 1 ? checksum64(host, h->data_bytes) : file_checksum(*h, *m, host)) != h->checksum) {
      s = fail(GC_ERR_IO, "checkpoint: '" + path + "' fails its checksum");
    }
  }
  std::fclose(in);
  return s;
}

}  // namespace
}  // namespace gcb

// ---- asynchronous snapshots --------------------------------------------------
struct gc_snapshotter {
  gc_context* ctx = nullptr;
  cudaStream_t copy = nullptr;
  struct Slot {
    void* dev = nullptr;
    void* host = nullptr;
    size_t cap = 0;
    cudaEvent_t staged = nullptr;  // device copy done (on the context stream)
    cudaEvent_t landed = nullptr;  // host copy done (on the copy stream)
    bool busy = false;
  };
  std::vector<Slot> slots;
  int next = 0;
  struct Job {
    int slot;
    bool vtk;
    gc_grid g;
    gc_dtype dt;
    int comps;
    gc_vtk_encoding enc;
    std::string path, text;  // text: field name (VTK) or metadata (checkpoint)
  };
  std::deque<Job> jobs;
  std::mutex mu;
  std::condition_variable cv;
  std::string error;  // first failure of the writer thread
  bool stop = false;
  std::thread writer;
};

namespace gcb {
namespace {

void writer_loop(gc_snapshotter* s) {
  cudaSetDevice(s->ctx->device);
  for (;;) {
    gc_snapshotter::Job job;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv.wait(lock, [&] { return s->stop || !s->jobs.empty(); });
      if (s->jobs.empty()) return;
      job = s->jobs.front();
    }
    gc_snapshotter::Slot& slot = s->slots[job.slot];
    std::string err;
    const cudaError_t e = cudaEventSynchronize(slot.landed);
    if (e != cudaSuccess) {
      err = std::string("snapshot: copy to the host failed: ") + cudaGetErrorString(e);
    } else {
      const gc_status st = job.vtk ? write_vtk_file(&job.g, job.dt, slot.host, job.path, job.text, job.enc)
                                   : write_ckpt_file(&job.g, job.dt, job.comps, slot.host, job.path, job.text);
      if (st != GC_OK) err = gc_last_error();
    }
    {
      std::lock_guard<std::mutex> lock(s->mu);
      if (!err.empty() && s->error.empty()) s->error = err;
      slot.busy = false;
      s->jobs.pop_front();
    }
    s->cv.notify_all();
  }
}

gc_status enqueue(gc_snapshotter* s, const gc_grid* g, gc_dtype dt, int comps, const void* field, bool vtk,
                  const char* path, const char* text, gc_vtk_encoding enc) {
  if (!s) return fail(GC_ERR_INVALID_ARG, "snapshot: null snapshotter");
  Call call(s->ctx);
  gc_status st = call.st;
  if (st != GC_OK) return st;
  if ((st = check_grid(g)) != GC_OK) return st;
  if (!field || !path) return fail(GC_ERR_INVALID_ARG, "snapshot: null pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "snapshot: unknown dtype");
  if (comps < 1) return fail(GC_ERR_INVALID_ARG, "snapshot: components must be >= 1");
  const size_t bytes = cells(g) * static_cast<size_t>(comps) * dtype_size(dt);
  gc_snapshotter::Slot* slot;
  int index;
  {
    std::unique_lock<std::mutex> lock(s->mu);
    index = s->next;
    slot = &s->slots[index];
    s->cv.wait(lock, [&] { return !slot->busy; });
    if (!s->error.empty()) return fail(GC_ERR_IO, s->error);
  }
  s->next = (s->next + 1) % static_cast<int>(s->slots.size());
  if (slot->cap < bytes) {
    if (slot->dev) cudaFree(slot->dev);
    if (slot->host) cudaFreeHost(slot->host);
    slot->dev = slot->host = nullptr;
    slot->cap = 0;
    GC_CUDA(cudaMalloc(&slot->dev, bytes));
    GC_CUDA(cudaHostAlloc(&slot->host, bytes, cudaHostAllocDefault));
    slot->cap = bytes;
  }
  GC_CUDA(cudaMemcpyAsync(slot->dev, field, bytes, cudaMemcpyDeviceToDevice, s->ctx->stream));
  GC_CUDA(cudaEventRecord(slot->staged, s->ctx->stream));
  GC_CUDA(cudaStreamWaitEvent(s->copy, slot->staged, 0));
  GC_CUDA(cudaMemcpyAsync(slot->host, slot->dev, bytes, cudaMemcpyDeviceToHost, s->copy));
  GC_CUDA(cudaEventRecord(slot->landed, s->copy));
  {
    std::lock_guard<std::mutex> lock(s->mu);
    slot->busy = true;
    s->jobs.push_back(gc_snapshotter::Job{index, vtk, *g, dt, comps, enc, path, text ? text : ""});
  }
  s->cv.notify_all();
  return GC_OK;
}

}  // namespace
}  // namespace gcb

using namespace gcb;

extern "C" {

GC_API gc_status gc_write_vtk(const gc_grid* g, gc_dtype dt, const void* host, const char* path, const char* field_name,
                              gc_vtk_encoding enc) {
  gc_status s = check_grid(g);
  if (s != GC_OK) return s;
  if (!host || !path || !field_name) return fail(GC_ERR_INVALID_ARG, "writeVtkStructuredPoints: null pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "writeVtkStructuredPoints: unknown dtype");
  if (enc != GC_VTK_ASCII && enc != GC_VTK_BINARY) return fail(GC_ERR_INVALID_ARG, "writeVtkStructuredPoints: unknown encoding");
  return write_vtk_file(g, dt, host, path, field_name, enc);
}

GC_API gc_status gc_write_checkpoint(const gc_grid* g, gc_dtype dt, int32_t components, const void* host,
                                     const char* path, const char* meta_json) {
  gc_status s = check_grid(g);
  if (s != GC_OK) return s;
  if (!host || !path) return fail(GC_ERR_INVALID_ARG, "checkpoint: null pointer");
  if (dt != GC_F64 && dt != GC_F32) return fail(GC_ERR_INVALID_ARG, "checkpoint: unknown dtype");
  if (components < 1) return fail(GC_ERR_INVALID_ARG, "checkpoint: components must be >= 1");
  return write_ckpt_file(g, dt, components, host, path, meta_json ? meta_json : "");
}

GC_API gc_status gc_checkpoint_info(const char* path, gc_grid* g, gc_dtype* dt, int32_t* components,
                                    size_t* meta_len) {
  if (!path) return fail(GC_ERR_INVALID_ARG, "checkpoint: null path");
  std::FILE* in = std::fopen(path, "rb");
  if (!in) return fail(GC_ERR_IO, std::string("checkpoint: cannot open '") + path + "'");
  CkptHeader h;
  const gc_status s = read_ckpt_header(in, path, &h);
  std::fclose(in);
  if (s != GC_OK) return s;
  if (g) *g = gc_grid{h.nx, h.ny, h.nz, h.hx, h.hy, h.hz};
  if (dt) *dt = static_cast<gc_dtype>(h.dtype);
  if (components) *components = h.components;
  if (meta_len) *meta_len = static_cast<size_t>(h.meta_len);
  return GC_OK;
}

GC_API gc_status gc_read_checkpoint(const char* path, void* host, size_t host_bytes, char* meta, size_t meta_cap) {
  if (!path || !host) return fail(GC_ERR_INVALID_ARG, "checkpoint: null pointer");
  CkptHeader h;
  std::string m;
  const gc_status s = read_ckpt(path, &h, &m, host, host_bytes);
  if (s != GC_OK) return s;
  if (meta && meta_cap) {
    const size_t n = std::min(meta_cap - 1, m.size());
    std::memcpy(meta, m.data(), n);
    meta[n] = '\0';
  }
  return GC_OK;
}

GC_API gc_status gc_load_checkpoint(gc_context* ctx, const char* path, void* field, size_t field_bytes, char* meta,
                                    size_t meta_cap) {
  Call call(ctx);
  gc_status s = call.st;
  if (s != GC_OK) return s;
  if (!path || !field) return fail(GC_ERR_INVALID_ARG, "checkpoint: null pointer");
  size_t meta_len = 0;
  gc_grid g;
  gc_dtype dt;
  int32_t comps;
  if ((s = gc_checkpoint_info(path, &g, &dt, &comps, &meta_len)) != GC_OK) return s;
  const size_t bytes = cells(&g) * static_cast<size_t>(comps) * dtype_size(dt);
  if (field_bytes < bytes)
    return fail(GC_ERR_INVALID_ARG, "checkpoint: device buffer of " + std::to_string(field_bytes) +
                                        " bytes, field has " + std::to_string(bytes));
  void* host = nullptr;
  GC_CUDA(cudaHostAlloc(&host, bytes ? bytes : 1, cudaHostAllocDefault));
  s = gc_read_checkpoint(path, host, bytes, meta, meta_cap);
  if (s == GC_OK) {
    cudaError_t e = cudaMemcpyAsync(field, host, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) s = fail(GC_ERR_CUDA, std::string("checkpoint: copy to the device failed: ") + cudaGetErrorString(e));
  }
  cudaFreeHost(host);
  return s;
}

GC_API gc_status gc_snapshotter_create(gc_context* ctx, int32_t depth, gc_snapshotter** out) {
  gc_status s = check_ctx(ctx);
  if (s != GC_OK) return s;
  if (!out) return fail(GC_ERR_INVALID_ARG, "snapshot: null output pointer");
  if (depth < 1 || depth > 16) return fail(GC_ERR_INVALID_ARG, "snapshot: depth must be 1..16");
  auto* sn = new gc_snapshotter();
  sn->ctx = ctx;
  sn->slots.resize(static_cast<size_t>(depth));
  cudaError_t e = cudaStreamCreateWithFlags(&sn->copy, cudaStreamNonBlocking);
  for (auto& slot : sn->slots) {
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.staged, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.landed, cudaEventDisableTiming | cudaEventBlockingSync);
  }
  if (e != cudaSuccess) {
    gc_snapshotter_destroy(sn);
    return fail(GC_ERR_CUDA, std::string("snapshot: ") + cudaGetErrorString(e));
  }
  sn->writer = std::thread(writer_loop, sn);
  *out = sn;
  return GC_OK;
}

GC_API gc_status gc_snapshot_vtk(gc_snapshotter* s, const gc_grid* g, gc_dtype dt, const void* field, const char* path,
                                 const char* field_name, gc_vtk_encoding enc) {
  if (enc != GC_VTK_ASCII && enc != GC_VTK_BINARY) return fail(GC_ERR_INVALID_ARG, "snapshot: unknown encoding");
  if (!field_name) return fail(GC_ERR_INVALID_ARG, "snapshot: null field name");
  return enqueue(s, g, dt, 1, field, true, path, field_name, enc);
}

GC_API gc_status gc_snapshot_checkpoint(gc_snapshotter* s, const gc_grid* g, gc_dtype dt, int32_t components,
                                        const void* field, const char* path, const char* meta_json) {
  return enqueue(s, g, dt, components, field, false, path, meta_json, GC_VTK_ASCII);
}

GC_API gc_status gc_snapshotter_flush(gc_snapshotter* s) {
  if (!s) return fail(GC_ERR_INVALID_ARG, "snapshot: null snapshotter");
  std::unique_lock<std::mutex> lock(s->mu);
  s->cv.wait(lock, [&] { return s->jobs.empty(); });
  if (!s->error.empty()) {
    const std::string e = s->error;
    s->error.clear();
    return fail(GC_ERR_IO, e);
  }
  return GC_OK;
}

GC_API gc_status gc_snapshotter_destroy(gc_snapshotter* s) {
  if (!s) return GC_OK;
  gc_status st = GC_OK;
  if (s->writer.joinable()) {
    st = gc_snapshotter_flush(s);
    {
      std::lock_guard<std::mutex> lock(s->mu);
      s->stop = true;
    }
    s->cv.notify_all();
    s->writer.join();
  }
  for (auto& slot : s->slots) {
    if (slot.dev) cudaFree(slot.dev);
    if (slot.host) cudaFreeHost(slot.host);
    if (slot.staged) cudaEventDestroy(slot.staged);
    if (slot.landed) cudaEventDestroy(slot.landed);
  }
  if (s->copy) cudaStreamDestroy(s->copy);
  delete s;
  return st;
}

}  // extern "C"
