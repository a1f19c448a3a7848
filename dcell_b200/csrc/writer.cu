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
// A device write snapshots the data into a device staging buffer on the
// caller's stream (HBM to HBM), then a copy stream of the writer moves it to
// pinned host memory while the caller's stream runs on; a writer thread waits
// for each copy, converts and writes the file.  Host writes copy into pinned
// memory and go through the same thread.  dcell_writer_flush waits for every
// pending write and returns the first error.
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

enum JobKind { JOB_GRID, JOB_NODES, JOB_PARTICLES };

struct Job {
  JobKind kind;
  std::string path;       // main file
  std::string info;       // .info companion ("" for none)
  int dof = 1;            // grid block size
  int dim = 3;            // nodes: 2 or 3
  int dtype = DCELL_F64;  // grid / particles element type
  long long count = 0;    // values (grid), records (particles); nodes: capacity
  std::string pos_path, size_path, pos_line, size_line;  // grid: appended lines
  std::vector<unsigned char> host;  // host data (host writes)
  void *pinned = nullptr;           // pinned data (device writes), from the pool
  size_t pinned_cap = 0;
  size_t bytes = 0;
  void *staging = nullptr;          // device staging buffer, from the pool
  size_t staging_cap = 0;
  cudaEvent_t done = nullptr;       // copy completion (device writes)
};

// Reusable buffers (device staging, pinned host): a buffer is taken when it
// holds the request and at most twice it, else a new one is allocated.
struct BufPool {
  std::multimap<size_t, void *> free_;
  bool device;
  explicit BufPool(bool dev) : device(dev) {}
  void *take(size_t bytes, size_t &cap) {
    auto it = free_.lower_bound(bytes);
    if (it != free_.end() && it->first <= 2 * bytes + 4096) {
      void *p = it->second;
      cap = it->first;
      free_.erase(it);
      return p;
    }
    void *p = nullptr;
    const cudaError_t e = device ? cudaMalloc(&p, bytes) : cudaMallocHost(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    cap = bytes;
    return p;
  }
  void give(void *p, size_t cap) {
    if (p) free_.emplace(cap, p);
  }
  void clear() {
    for (auto &kv : free_) device ? cudaFree(kv.second) : cudaFreeHost(kv.second);
    free_.clear();
  }
};

void put_be32(FILE *f, int32_t v) {
  unsigned char b[4] = {(unsigned char)(v >> 24), (unsigned char)(v >> 16), (unsigned char)(v >> 8), (unsigned char)v};
  fwrite(b, 1, 4, f);
}

// FP64 values, big-endian, in chunks
bool put_be64(FILE *f, const double *v, long long n) {
  unsigned char buf[8 * 1024];
  long long i = 0;
  while (i < n) {
    const long long m = (n - i) < 1024 ? (n - i) : 1024;
    for (long long k = 0; k < m; ++k) {
      uint64_t u;
      memcpy(&u, v + i + k, 8);
      for (int b = 0; b < 8; ++b) buf[8 * k + b] = (unsigned char)(u >> (56 - 8 * b));
    }
    if (fwrite(buf, 8, (size_t)m, f) != (size_t)m) return false;
    i += m;
  }
  return true;
}

}  // namespace

struct dcell_writer {
  std::string dir, tmpdir;
  int device = 0;
  bool cuda_ready = false;
  cudaStream_t copy = nullptr;
  std::mutex mu;
  std::condition_variable cv, idle;
  std::deque<std::unique_ptr<Job>> queue;
  int inflight = 0;
  bool stop = false;
  int error = DCELL_OK;
  std::string error_text;
  std::map<std::string, bool> opened;  // .pos/.size files truncated on first write
  std::mutex pool_mu;
  BufPool dev_pool{true}, host_pool{false};
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
      }
      idle.notify_all();
    }
  }

  void release(Job &j) {
    if (j.done) {
      cudaSetDevice(device);
      cudaEventDestroy(j.done);
      j.done = nullptr;
    }
    std::lock_guard<std::mutex> g(pool_mu);
    dev_pool.give(j.staging, j.staging_cap);
    host_pool.give(j.pinned, j.pinned_cap);
    j.staging = j.pinned = nullptr;
  }

  const unsigned char *data(Job &j) {
    if (j.done) {
      cudaSetDevice(device);
      if (cudaEventSynchronize(j.done) != cudaSuccess) {
        fail(DCELL_ERR_CUDA, "device-to-host copy of " + j.path + " failed");
        return nullptr;
      }
      return (const unsigned char *)j.pinned;
    }
    static const unsigned char empty = 0;
    return j.host.empty() ? &empty : j.host.data();
  }

  void process(Job &j) {
    const unsigned char *p = data(j);
    if (!p) return;
    FILE *f = fopen(j.path.c_str(), "wb");
    if (!f) {
      fail(DCELL_ERR_ARG, "cannot open " + j.path + ": " + strerror(errno));
      return;
    }
    bool ok = true;
    std::vector<double> tmp;
    if (j.kind == JOB_GRID) {
      const double *v = (const double *)p;
      if (j.dtype == DCELL_F32) {
        tmp.resize((size_t)j.count);
        for (long long i = 0; i < j.count; ++i) tmp[i] = ((const float *)p)[i];
        v = tmp.data();
      }
      put_be32(f, VEC_FILE_CLASSID);
      put_be32(f, (int32_t)j.count);
      ok = put_be64(f, v, j.count);
    } else if (j.kind == JOB_NODES) {
      const dcell_irregular_node *nodes = (const dcell_irregular_node *)p;
      int32_t cnt;
      memcpy(&cnt, p + j.bytes - sizeof(int32_t), sizeof(int32_t));
      const long long n = cnt < j.count ? cnt : j.count;
      for (long long i = 0; i < n && ok; ++i) {
        const dcell_irregular_node &q = nodes[i];
        double row[23] = {0};
        if (j.dim == 2) {
          if (q.axis == -1) continue;
          // X, pos, n, f1, fa1, k, f1_n, f1_nn (IrregularNodes.c:159-169)
          row[0] = q.X[0], row[1] = q.X[1], row[2] = q.pos[0], row[3] = q.pos[1], row[4] = q.n[0], row[5] = q.n[1];
          row[8] = q.k;
          ok = put_be64(f, row, 11);
        } else {
          // X, pos, n, k, then the IIM quantities (IrregularNodes.c:190-212)
          row[0] = q.X[0], row[1] = q.X[1], row[2] = q.X[2], row[3] = q.pos[0], row[4] = q.pos[1],
          row[5] = q.pos[2], row[6] = q.n[0], row[7] = q.n[1], row[8] = q.n[2], row[9] = q.k;
          ok = put_be64(f, row, 23);
        }
      }
    } else {
      const double *v = (const double *)p;
      if (j.dtype == DCELL_F32) {
        tmp.resize((size_t)j.count * 4);
        for (long long i = 0; i < 4 * j.count; ++i) tmp[i] = ((const float *)p)[i];
        v = tmp.data();
      }
      ok = fwrite(v, sizeof(double) * 4, (size_t)j.count, f) == (size_t)j.count;
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
      fail(DCELL_ERR_ARG, "writing " + j.path + " failed");
      return;
    }
    if (!j.info.empty() || j.kind != JOB_PARTICLES) {
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
    cuda_ready = true;
    return DCELL_OK;
  }

  // Snapshot `bytes` of device data (plus an optional trailing device int)
  // and queue its copy to pinned memory.
  int stage_device(Job &j, const void *src, size_t bytes, const int *tail, cudaStream_t st) {
    int rc = ensure_cuda();
    if (rc) return rc;
    const size_t total = bytes + (tail ? sizeof(int32_t) : 0);
    j.bytes = total;
    {
      std::lock_guard<std::mutex> g(pool_mu);
      j.staging = dev_pool.take(total > 0 ? total : 1, j.staging_cap);
      j.pinned = j.staging ? host_pool.take(total > 0 ? total : 1, j.pinned_cap) : nullptr;
    }
    if (!j.staging || !j.pinned) {
      dcell_set_error(DCELL_ERR_NOMEM, "staging or pinned buffer of %zu bytes", total);
      return DCELL_ERR_NOMEM;
    }
    cudaEvent_t snap;
    DCELL_CUDA_CHECK(cudaEventCreateWithFlags(&snap, cudaEventDisableTiming));
    DCELL_CUDA_CHECK(cudaEventCreateWithFlags(&j.done, cudaEventDisableTiming));
    if (bytes) DCELL_CUDA_CHECK(cudaMemcpyAsync(j.staging, src, bytes, cudaMemcpyDeviceToDevice, st));
    if (tail)
      DCELL_CUDA_CHECK(cudaMemcpyAsync((char *)j.staging + bytes, tail, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    DCELL_CUDA_CHECK(cudaEventRecord(snap, st));
    DCELL_CUDA_CHECK(cudaStreamWaitEvent(copy, snap, 0));
    DCELL_CUDA_CHECK(cudaMemcpyAsync(j.pinned, j.staging, total, cudaMemcpyDeviceToHost, copy));
    DCELL_CUDA_CHECK(cudaEventRecord(j.done, copy));
    cudaEventDestroy(snap);
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
    cudaStreamDestroy(w->copy);
    w->dev_pool.clear();
    w->host_pool.clear();
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
  if ((rc = w->stage_device(*j, data, bytes, nullptr, (cudaStream_t)stream))) {
    w->release(*j);
    return rc;
  }
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
  if ((rc = w->stage_device(*j, nodes, (size_t)capacity * sizeof(dcell_irregular_node), count, (cudaStream_t)stream))) {
    w->release(*j);
    return rc;
  }
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
                            (cudaStream_t)stream))) {
    w->release(*j);
    return rc;
  }
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
