// On-disk output of the level-set path in the reference's formats, written
// asynchronously from device memory.
//
//   grid       <dir>/<name>.<t+10000>.Real64 (+ .info), and one line per write
//              appended to <dir>/<name>.pos and <dir>/<name>.size -- GridWrite
//              (Common/Serialize.c:23-55): PETSc's binary Vec format, i.e. the
//              int32 class id 1211214, the int32 length, then the FP64 values,
//              all big-endian; the .info companion carries
//              "-vecload_block_size <dof>" when dof > 1.
//   nodes      <dir>/<name>.irregNode.<idx+10000>.array --
//              LevelSetWriteIrregularNodeList (LevelSetMethod/IrregularNodes.c:
//              145-246): rows of big-endian FP64, 11 per 2D node with
//              axis != -1, 23 per 3D node; the IIM quantities this path does
//              not compute are 0, as in the reference's zeroed nodes.
//   particles  <tmpdir>/<name>.<t+10000>.array -- ArrayWrite (Common/Array.c:
//              133-150): the raw records (X.x, X.y, X.z, radius as native
//              FP64).
//
// A device write snapshots the data on the caller's stream into memory from
// the writer's stream-ordered pool (HBM to HBM: the only cost the caller's
// stream sees); the writer thread moves each snapshot through two pinned
// 60 MiB chunks on its own copy stream (the copy of one chunk overlaps the
// formatting and writing of the other) and frees it.  The staged total is
// bounded (DCELL_WRITER_MAX_STAGED_MB, default 16 GiB): a write waits while
// it would exceed it.  Host writes keep a copy of the data and go through the
// same thread.  dcell_writer_flush waits for every pending write and returns
// the first error.
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dcell_common.cuh"
#include "dcell_kernels.h"

namespace {

constexpr int FILE_COUNT_START = 10000;  // Common/Common.h:59
constexpr int32_t VEC_FILE_CLASSID = 1211214;
// pinned chunk: a multiple of every record size (4, 8, 16, 32, 120 bytes)
constexpr size_t CHUNK = 480u << 17;  // 60 MiB
constexpr size_t DEFAULT_MAX_STAGED = 16ull << 30;

enum JobKind { JOB_GRID, JOB_NODES, JOB_PARTICLES };

struct Job {
  JobKind kind;
  std::string path;       // main file
  std::string info;       // .info companion ("" for none)
  int dof = 1;            // grid block size
  int dim = 3;            // nodes: 2 or 3
  int dtype = DCELL_F64;  // grid / particles element type
  long long count = 0;    // values (grid), records (particles / nodes; nodes: capacity)
  std::string pos_path, size_path, pos_line, size_line;  // grid: appended lines
  std::vector<unsigned char> host;  // host writes: the data (nodes: records + int32 count)
  void *staging = nullptr;          // device writes: stream-ordered snapshot
  size_t bytes = 0;                 // staged bytes (nodes: records + int32 count)
  cudaEvent_t snap = nullptr;       // snapshot complete on the caller's stream
};

void be32(unsigned char *o, int32_t v) {
  o[0] = (unsigned char)(v >> 24), o[1] = (unsigned char)(v >> 16), o[2] = (unsigned char)(v >> 8),
  o[3] = (unsigned char)v;
}

void be64(unsigned char *o, double d) {
  uint64_t u;
  memcpy(&u, &d, 8);
  for (int b = 0; b < 8; ++b) o[b] = (unsigned char)(u >> (56 - 8 * b));
}

}  // namespace

struct dcell_writer {
  std::string dir, tmpdir;
  int device = 0;
  bool cuda_ready = false;
  cudaStream_t copy = nullptr;
  cudaMemPool_t pool = nullptr;
  void *pin[2] = {nullptr, nullptr};
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  std::mutex mu;
  std::condition_variable cv, idle;
  std::deque<std::unique_ptr<Job>> queue;
  int inflight = 0;
  size_t staged = 0, max_staged = DEFAULT_MAX_STAGED;
  bool stop = false;
  int error = DCELL_OK;
  std::string error_text;
  std::map<std::string, bool> opened;  // .pos/.size files truncated on first write
  std::vector<unsigned char> out;      // formatted bytes of one chunk
  std::thread thread;

  void fail(int code, const std::string &text) {
    std::lock_guard<std::mutex> g(mu);
    if (!error) {
      error = code;
      error_text = text;
    }
  }

  void run() {
    for (;;) {
      std::unique_ptr<Job> job;
      {
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&] { return stop || !queue.empty(); });
        if (queue.empty()) return;
        job = std::move(queue.front());
        queue.pop_front();
      }
      process(*job);
      release(*job);
      {
        std::lock_guard<std::mutex> g(mu);
        --inflight;
        staged -= job->staging ? job->bytes : 0;
      }
      idle.notify_all();
    }
  }

  void release(Job &j) {
    if (!j.snap) return;
    cudaSetDevice(device);
    // order the free after the snapshot copy on the caller's stream, also
    // when process() gave up before drain() made the copy stream wait for it
    cudaStreamWaitEvent(copy, j.snap, 0);
    cudaFreeAsync(j.staging, copy);
    cudaEventDestroy(j.snap);
    j.snap = nullptr;
  }

  // Feed the job's first `bytes` bytes to sink in pieces of whole records:
  // host data at once, device data through the two pinned chunks (the copy of
  // one overlaps the formatting of the other).
  template <typename Sink>
  bool drain(Job &j, size_t bytes, Sink sink) {
    if (!j.snap) return bytes == 0 || sink(j.host.data(), bytes);
    cudaSetDevice(device);
    if (!ensure_pins() || cudaStreamWaitEvent(copy, j.snap, 0) != cudaSuccess) return false;
    const size_t nchunk = (bytes + CHUNK - 1) / CHUNK;
    size_t prev_len = 0;
    for (size_t c = 0; c <= nchunk; ++c) {
      if (c < nchunk) {
        const size_t off = c * CHUNK, len = bytes - off < CHUNK ? bytes - off : CHUNK;
        if (cudaMemcpyAsync(pin[c & 1], (const char *)j.staging + off, len, cudaMemcpyDeviceToHost, copy) !=
                cudaSuccess ||
            cudaEventRecord(pin_ev[c & 1], copy) != cudaSuccess)
          return false;
        if (c == 0) {
          prev_len = len;
          continue;
        }
        if (cudaEventSynchronize(pin_ev[(c - 1) & 1]) != cudaSuccess) return false;
        if (!sink((const unsigned char *)pin[(c - 1) & 1], prev_len)) return false;
        prev_len = len;
      } else if (nchunk) {
        if (cudaEventSynchronize(pin_ev[(c - 1) & 1]) != cudaSuccess) return false;
        if (!sink((const unsigned char *)pin[(c - 1) & 1], prev_len)) return false;
      }
    }
    return true;
  }

  // The node count stored after the records.
  bool node_count(Job &j, int32_t &cnt) {
    if (!j.snap) {
      memcpy(&cnt, j.host.data() + j.bytes - sizeof(int32_t), sizeof cnt);
      return true;
    }
    cudaSetDevice(device);
    if (!ensure_pins() || cudaStreamWaitEvent(copy, j.snap, 0) != cudaSuccess ||
        cudaMemcpyAsync(pin[0], (const char *)j.staging + j.bytes - sizeof(int32_t), sizeof(int32_t),
                        cudaMemcpyDeviceToHost, copy) != cudaSuccess ||
        cudaStreamSynchronize(copy) != cudaSuccess)
      return false;
    memcpy(&cnt, pin[0], sizeof cnt);
    return true;
  }

  bool ensure_pins() {
    if (pin[0]) return true;
    for (int k = 0; k < 2; ++k) {
      if (cudaMallocHost(&pin[k], CHUNK) != cudaSuccess ||
          cudaEventCreateWithFlags(&pin_ev[k], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        fail(DCELL_ERR_NOMEM, "pinned staging of the writer");
        return false;
      }
    }
    return true;
  }

  void process(Job &j) {
    FILE *f = fopen(j.path.c_str(), "wb");
    if (!f) {
      fail(DCELL_ERR_ARG, "cannot open " + j.path + ": " + strerror(errno));
      return;
    }
    bool ok = true;
    const size_t el = j.dtype == DCELL_F64 ? 8 : 4;
    if (j.kind == JOB_GRID) {
      unsigned char head[8];
      be32(head, VEC_FILE_CLASSID);
      be32(head + 4, (int32_t)j.count);
      ok = fwrite(head, 1, 8, f) == 8;
      ok = ok && drain(j, (size_t)j.count * el, [&](const unsigned char *p, size_t n) {
             const size_t m = n / el;
             out.resize(m * 8);
             for (size_t i = 0; i < m; ++i) {
               double v;
               if (el == 8)
                 memcpy(&v, p + 8 * i, 8);
               else {
                 float x;
                 memcpy(&x, p + 4 * i, 4);
                 v = x;
               }
               be64(out.data() + 8 * i, v);
             }
             return fwrite(out.data(), 1, out.size(), f) == out.size();
           });
    } else if (j.kind == JOB_NODES) {
      int32_t cnt = 0;
      ok = node_count(j, cnt);
      const long long n = cnt < 0 ? 0 : (cnt < j.count ? cnt : j.count);
      ok = ok && drain(j, (size_t)n * sizeof(dcell_irregular_node), [&](const unsigned char *p, size_t nb) {
             const size_t m = nb / sizeof(dcell_irregular_node);
             out.resize(m * 23 * 8);
             size_t o = 0;
             for (size_t i = 0; i < m; ++i) {
               dcell_irregular_node q;
               memcpy(&q, p + i * sizeof q, sizeof q);
               double row[23] = {0};
               int w = 23;
               if (j.dim == 2) {
                 if (q.axis == -1) continue;
                 // X, pos, n, f1, fa1, k, f1_n, f1_nn (IrregularNodes.c:159-169)
                 row[0] = q.X[0], row[1] = q.X[1], row[2] = q.pos[0], row[3] = q.pos[1], row[4] = q.n[0],
                 row[5] = q.n[1], row[8] = q.k;
                 w = 11;
               } else {
                 // X, pos, n, k, then the IIM quantities (IrregularNodes.c:190-212)
                 row[0] = q.X[0], row[1] = q.X[1], row[2] = q.X[2], row[3] = q.pos[0], row[4] = q.pos[1],
                 row[5] = q.pos[2], row[6] = q.n[0], row[7] = q.n[1], row[8] = q.n[2], row[9] = q.k;
               }
               for (int k = 0; k < w; ++k) be64(out.data() + o + 8 * k, row[k]);
               o += 8 * w;
             }
             return fwrite(out.data(), 1, o, f) == o;
           });
    } else {
      ok = drain(j, (size_t)j.count * 4 * el, [&](const unsigned char *p, size_t n) {
        if (el == 8) return fwrite(p, 1, n, f) == n;
        const size_t m = n / 4;
        out.resize(m * 8);
        for (size_t i = 0; i < m; ++i) {
          float x;
          memcpy(&x, p + 4 * i, 4);
          const double v = x;
          memcpy(out.data() + 8 * i, &v, 8);
        }
        return fwrite(out.data(), 1, out.size(), f) == out.size();
      });
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
      fail(DCELL_ERR_ARG, "writing " + j.path + " failed");
      return;
    }
    if (j.kind != JOB_PARTICLES) {  // PetscViewerBinaryOpen's .info companion
      FILE *fi = fopen((j.path + ".info").c_str(), "wb");
      if (!fi) {
        fail(DCELL_ERR_ARG, "cannot open " + j.path + ".info");
        return;
      }
      if (!j.info.empty()) fputs(j.info.c_str(), fi);
      fclose(fi);
    }
    if (j.kind == JOB_GRID) {
      for (int k = 0; k < 2; ++k) {
        const std::string &path = k ? j.size_path : j.pos_path;
        const bool first = !opened[path];
        opened[path] = true;
        FILE *fa = fopen(path.c_str(), first ? "w" : "a");
        if (!fa) {
          fail(DCELL_ERR_ARG, "cannot open " + path);
          return;
        }
        fputs((k ? j.size_line : j.pos_line).c_str(), fa);
        fclose(fa);
      }
    }
  }

  int enqueue(std::unique_ptr<Job> job) {
    {
      std::lock_guard<std::mutex> g(mu);
      ++inflight;
      queue.push_back(std::move(job));
    }
    cv.notify_one();
    return DCELL_OK;
  }

  int ensure_cuda() {
    if (cuda_ready) return DCELL_OK;
    DCELL_CUDA_CHECK(cudaSetDevice(device));
    DCELL_CUDA_CHECK(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    DCELL_CUDA_CHECK(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = UINT64_MAX;  // keep freed snapshots for reuse
    DCELL_CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    const char *m = getenv("DCELL_WRITER_MAX_STAGED_MB");
    if (m && atoll(m) > 0) max_staged = (size_t)atoll(m) << 20;
    cuda_ready = true;
    return DCELL_OK;
  }

  // Snapshot `bytes` of device data (and an optional trailing device int32)
  // on the caller's stream; waits first while the staged total would exceed
  // the limit (the writer thread drains to disk).
  int stage_device(Job &j, const void *src, size_t bytes, const int *tail, cudaStream_t st) {
    int rc = ensure_cuda();
    if (rc) return rc;
    const size_t total = bytes + (tail ? sizeof(int32_t) : 0);
    j.bytes = total;
    {
      std::unique_lock<std::mutex> g(mu);
      idle.wait(g, [&] { return staged == 0 || staged + total <= max_staged; });
      staged += total;
    }
    if (cudaMallocFromPoolAsync(&j.staging, total > 0 ? total : 1, pool, st) != cudaSuccess) {
      cudaGetLastError();
      std::lock_guard<std::mutex> g(mu);
      staged -= total;
      j.staging = nullptr;
      dcell_set_error(DCELL_ERR_NOMEM, "snapshot of %zu bytes", total);
      return DCELL_ERR_NOMEM;
    }
    cudaError_t e = cudaEventCreateWithFlags(&j.snap, cudaEventDisableTiming);
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(j.staging, src, bytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && tail)
      e = cudaMemcpyAsync((char *)j.staging + bytes, tail, sizeof(int32_t), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(j.snap, st);
    if (e != cudaSuccess) {
      cudaFreeAsync(j.staging, st);
      if (j.snap) cudaEventDestroy(j.snap);
      j.snap = nullptr;
      j.staging = nullptr;
      std::lock_guard<std::mutex> g(mu);
      staged -= total;
      dcell_set_error(DCELL_ERR_CUDA, "snapshot for %s: %s", j.path.c_str(), cudaGetErrorString(e));
      return DCELL_ERR_CUDA;
    }
    return DCELL_OK;
  }
};

static std::string grid_file(dcell_writer *w, const char *name, int t, std::string suffix) {
  return w->dir + "/" + name + "." + std::to_string(t + FILE_COUNT_START) + suffix;
}

static int check_writer(dcell_writer *w, const char *name) {
  if (!w) {
    dcell_set_error(DCELL_ERR_ARG, "writer is NULL");
    return DCELL_ERR_ARG;
  }
  if (!name || !*name || strchr(name, '/')) {
    dcell_set_error(DCELL_ERR_ARG, "a plain file name is required");
    return DCELL_ERR_ARG;
  }
  return DCELL_OK;
}

static std::unique_ptr<Job> grid_job(dcell_writer *w, const char *name, int t, const dcell_geom *g, int dof,
                                     int dtype) {
  std::unique_ptr<Job> j(new Job());
  const bool is2d = g->n[2] < 2;
  const long long pts = (long long)g->n[0] * g->n[1] * (is2d ? 1 : g->n[2]);
  j->kind = JOB_GRID;
  j->path = grid_file(w, name, t, ".Real64");
  j->dof = dof;
  j->dtype = dtype;
  j->count = pts * dof;
  if (dof > 1) j->info = "-vecload_block_size " + std::to_string(dof) + "\n";
  j->pos_path = w->dir + "/" + name + ".pos";
  j->size_path = w->dir + "/" + name + ".size";
  char line[128];
  if (is2d) {
    snprintf(line, sizeof line, "%d %d\n", g->p[0], g->p[1]);
    j->pos_line = line;
    snprintf(line, sizeof line, "%d %d\n", g->n[0], g->n[1]);
    j->size_line = line;
  } else {
    snprintf(line, sizeof line, "%d %d %d\n", g->p[0], g->p[1], g->p[2]);
    j->pos_line = line;
    snprintf(line, sizeof line, "%d %d %d\n", g->n[0], g->n[1], g->n[2]);
    j->size_line = line;
  }
  return j;
}

static int check_grid_args(dcell_writer *w, const char *name, const dcell_geom *g, int dof, int dtype,
                           const void *data) {
  int rc = check_writer(w, name);
  if (rc) return rc;
  if (!g || g->n[0] < 1 || g->n[1] < 1 || g->n[2] < 0 || dof < 1 || !data ||
      (dtype != DCELL_F32 && dtype != DCELL_F64)) {
    dcell_set_error(DCELL_ERR_ARG, "geometry, dof >= 1, dtype and data are required");
    return DCELL_ERR_ARG;
  }
  const long long n = (long long)g->n[0] * g->n[1] * (g->n[2] < 2 ? 1 : g->n[2]) * dof;
  if (n >= (1LL << 31)) {
    dcell_set_error(DCELL_ERR_ARG, "the PETSc binary header holds at most 2^31 - 1 values");
    return DCELL_ERR_ARG;
  }
  return DCELL_OK;
}

extern "C" {

DCELL_API int dcell_writer_create(const char *dir, const char *tmpdir, int device, dcell_writer **out) {
  if (!dir || !out) {
    dcell_set_error(DCELL_ERR_ARG, "dir and out are required");
    return DCELL_ERR_ARG;
  }
  dcell_writer *w = new dcell_writer();
  w->dir = dir;
  const char *t = tmpdir ? tmpdir : getenv("PETSC_TMP");
  w->tmpdir = t ? t : "/tmp";
  w->device = device;
  w->thread = std::thread([w] { w->run(); });
  *out = w;
  return DCELL_OK;
}

DCELL_API int dcell_writer_flush(dcell_writer *w) {
  if (!w) {
    dcell_set_error(DCELL_ERR_ARG, "writer is NULL");
    return DCELL_ERR_ARG;
  }
  std::unique_lock<std::mutex> g(w->mu);
  w->idle.wait(g, [&] { return w->inflight == 0; });
  if (w->error) {
    dcell_set_error(w->error, "%s", w->error_text.c_str());
    const int e = w->error;
    w->error = DCELL_OK;
    w->error_text.clear();
    return e;
  }
  return DCELL_OK;
}

DCELL_API int dcell_writer_destroy(dcell_writer *w) {
  if (!w) return DCELL_OK;
  const int rc = dcell_writer_flush(w);
  {
    std::lock_guard<std::mutex> g(w->mu);
    w->stop = true;
  }
  w->cv.notify_all();
  w->thread.join();
  if (w->cuda_ready) {
    cudaSetDevice(w->device);
    cudaStreamSynchronize(w->copy);
    for (int k = 0; k < 2; ++k) {
      if (w->pin[k]) cudaFreeHost(w->pin[k]);
      if (w->pin_ev[k]) cudaEventDestroy(w->pin_ev[k]);
    }
    cudaStreamDestroy(w->copy);
    cudaMemPoolDestroy(w->pool);
  }
  delete w;
  return rc;
}

DCELL_API int dcell_writer_grid(dcell_writer *w, const char *name, int t, const dcell_geom *g, int dof, int dtype,
                                const void *data, void *stream) {
  int rc = check_grid_args(w, name, g, dof, dtype, data);
  if (rc) return rc;
  std::unique_ptr<Job> j = grid_job(w, name, t, g, dof, dtype);
  const size_t bytes = (size_t)j->count * (dtype == DCELL_F64 ? 8 : 4);
  if ((rc = w->stage_device(*j, data, bytes, nullptr, (cudaStream_t)stream))) return rc;
  return w->enqueue(std::move(j));
}

DCELL_API int dcell_writer_grid_host(dcell_writer *w, const char *name, int t, const dcell_geom *g, int dof,
                                     const double *data) {
  int rc = check_grid_args(w, name, g, dof, DCELL_F64, data);
  if (rc) return rc;
  std::unique_ptr<Job> j = grid_job(w, name, t, g, dof, DCELL_F64);
  j->host.assign((const unsigned char *)data, (const unsigned char *)data + (size_t)j->count * 8);
  return w->enqueue(std::move(j));
}

DCELL_API int dcell_writer_irregular_nodes(dcell_writer *w, const char *name, int idx, int dim,
                                           const dcell_irregular_node *nodes, const int *count, int capacity,
                                           void *stream) {
  int rc = check_writer(w, name);
  if (rc) return rc;
  if ((dim != 2 && dim != 3) || !count || capacity < 0 || (capacity > 0 && !nodes)) {
    dcell_set_error(DCELL_ERR_ARG, "dim 2 or 3, count and the node buffer are required");
    return DCELL_ERR_ARG;
  }
  std::unique_ptr<Job> j(new Job());
  j->kind = JOB_NODES;
  j->dim = dim;
  j->count = capacity;
  j->path = w->dir + "/" + name + ".irregNode." + std::to_string(idx + FILE_COUNT_START) + ".array";
  if ((rc = w->stage_device(*j, nodes, (size_t)capacity * sizeof(dcell_irregular_node), count,
                            (cudaStream_t)stream)))
    return rc;
  return w->enqueue(std::move(j));
}

DCELL_API int dcell_writer_irregular_nodes_host(dcell_writer *w, const char *name, int idx, int dim,
                                                const dcell_irregular_node *nodes, int count) {
  int rc = check_writer(w, name);
  if (rc) return rc;
  if ((dim != 2 && dim != 3) || count < 0 || (count > 0 && !nodes)) {
    dcell_set_error(DCELL_ERR_ARG, "dim 2 or 3 and the nodes are required");
    return DCELL_ERR_ARG;
  }
  std::unique_ptr<Job> j(new Job());
  j->kind = JOB_NODES;
  j->dim = dim;
  j->count = count;
  j->path = w->dir + "/" + name + ".irregNode." + std::to_string(idx + FILE_COUNT_START) + ".array";
  const size_t bytes = (size_t)count * sizeof(dcell_irregular_node);
  j->host.resize(bytes + sizeof(int32_t));
  if (bytes) memcpy(j->host.data(), nodes, bytes);
  const int32_t c = count;
  memcpy(j->host.data() + bytes, &c, sizeof c);
  j->bytes = j->host.size();
  return w->enqueue(std::move(j));
}

DCELL_API int dcell_writer_particles(dcell_writer *w, const char *name, int t, const void *particles, long long n,
                                     int dtype, void *stream) {
  int rc = check_writer(w, name);
  if (rc) return rc;
  if (n < 0 || (n > 0 && !particles) || (dtype != DCELL_F32 && dtype != DCELL_F64)) {
    dcell_set_error(DCELL_ERR_ARG, "particles, n >= 0 and a dtype are required");
    return DCELL_ERR_ARG;
  }
  std::unique_ptr<Job> j(new Job());
  j->kind = JOB_PARTICLES;
  j->dtype = dtype;
  j->count = n;
  j->path = w->tmpdir + "/" + name + "." + std::to_string(t + FILE_COUNT_START) + ".array";
  if ((rc = w->stage_device(*j, particles, (size_t)n * 4 * (dtype == DCELL_F64 ? 8 : 4), nullptr,
                            (cudaStream_t)stream)))
    return rc;
  return w->enqueue(std::move(j));
}

DCELL_API int dcell_writer_particles_host(dcell_writer *w, const char *name, int t, const double *particles,
                                          long long n) {
  int rc = check_writer(w, name);
  if (rc) return rc;
  if (n < 0 || (n > 0 && !particles)) {
    dcell_set_error(DCELL_ERR_ARG, "particles and n >= 0 are required");
    return DCELL_ERR_ARG;
  }
  std::unique_ptr<Job> j(new Job());
  j->kind = JOB_PARTICLES;
  j->dtype = DCELL_F64;
  j->count = n;
  j->path = w->tmpdir + "/" + name + "." + std::to_string(t + FILE_COUNT_START) + ".array";
  j->host.assign((const unsigned char *)particles, (const unsigned char *)particles + (size_t)n * 32);
  return w->enqueue(std::move(j));
}

}  // extern "C"
