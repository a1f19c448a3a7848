// Internal launcher interface between the CUDA translation units and the
// C ABI (capi.cu).  Not part of the public header.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "dcell_common.cuh"

// 3-D tiled TMA map (zero fill out of bounds, no swizzle) over a row-major
// array (x fastest) of dx x dy x dz values of `elem` bytes; box bx x by x bz.
// False when the driver's encoder is unavailable or rejects the map.
bool make_tensor_map_3d(CUtensorMap *m, CUtensorMapDataType type, const void *base, uint64_t dx, uint64_t dy,
                        uint64_t dz, uint32_t bx, uint32_t by, uint32_t bz, uint32_t elem);

int launch_sl_linear(const dcell::Geom &g, int dtype, const void *phi0, const void *vel, double dt, const int *band,
                     long long npts, int backtrace, void *phi, int *flags, cudaStream_t st, bool gather = false);
// FP32 trilinear step (sl_lin.cu): TMA z-march on dense 3-D grids, gathers otherwise
int launch_sl_lin_f32(const dcell::Geom &g, const float *phi0, const float *vel, double dt, const int *band,
                      long long npts, int backtrace, float *phi, int *flags, cudaStream_t st, bool gather = false);
// gather: the global-gather form even where the brick-staged one applies
int launch_sl_cubic(const dcell::Geom &g, int dtype, const void *phi0, const void *vel, double dt, const int *band,
                    long long npts, int interp, int backtrace, void *phi, int *flags, cudaStream_t st,
                    bool gather = false);
int launch_sl_tc(const dcell::Geom &g, const float *phi0, const float *vel, double dt, const int *band,
                 long long npts, int backtrace, float *phi, int *flags, cudaStream_t st);

int launch_split_bf16(const float *phi, uint32_t *out, long long n, cudaStream_t st);
int launch_batch_brick(const dcell_cell *cells, const dcell_tile *bricks, int nbricks, const uint32_t *phi0s,
                       const float *vel, int backtrace, float *phi, uint32_t *phis, int *flags, cudaStream_t st);
// Padded-cell batches staged by TMA: tensor maps encoded on the host (two
// per cell, `out` holds 2 * ncells CUtensorMap), then the batched brick step.
int batch_tma_maps_host(const dcell_cell *cells, int ncells, const uint32_t *phi0s, const float *vel, void *out);
int launch_batch_brick_tma(const dcell_cell *cells, const dcell_tile *bricks, int nbricks, const void *maps,
                           const uint32_t *phi0s, const float *vel, int backtrace, float *phi, uint32_t *phis,
                           int *flags, cudaStream_t st);
// One z-slab of the dense split-state tensor-core step: z bricks [bz0, bz0 +
// nbz) of tc_slab_planes() planes each, gated on max |w| (FP32 bits at
// gate_maxw) * dt / h_z <= gate_limit.
struct TcSlab {
  int bz0, nbz;
  const int *gate_maxw;
  float gate_limit;
};
int tc_slab_planes();
bool tc_brick_applicable(const dcell::Geom &g, const void *phi0s, const void *vel);
// z bricks [slab.bz0, slab.bz0 + slab.nbz) of the dense split-state step,
// gated (see TcSlab); phis (nullable) receives the stepped split words
int launch_sl_tc_slab(const dcell::Geom &g, const uint32_t *phi0s, const float *vel, double dt, int backtrace,
                      float *phi, uint32_t *phis, int *flags, cudaStream_t st, const TcSlab &slab);
// z bricks [bz0, bz0 + nbz) of the dense split-state step (tc_slab_planes()
// planes each), no gate
int launch_sl_tc_split_planes(const dcell::Geom &g, const uint32_t *phi0s, const float *vel, double dt,
                              int backtrace, float *phi, uint32_t *phis, int *flags, cudaStream_t st, int bz0,
                              int nbz);
int launch_sl_tc_split(const dcell::Geom &g, const uint32_t *phi0s, const float *vel, double dt, const int *band,
                       long long npts, int backtrace, float *phi, uint32_t *phis, int *flags, cudaStream_t st);
int launch_batch_tc(const dcell_cell *cells, const dcell_tile *tiles, int ntiles, int tx, int ty, int ctas_per_sm,
                    const float *phi0, const float *vel, int backtrace, float *phi, int *flags, cudaStream_t st);
int launch_batch_cuda_core(const dcell_cell *cells, const dcell_tile *tiles, int ntiles, int tx, int ty, int tz,
                           int ctas_per_sm, const float *phi0, const float *vel, int interp, int backtrace, float *phi,
                           int *flags, cudaStream_t st);

int launch_sl_adjoint(const dcell::Geom &g, int dtype, const void *phi0, const void *vel, double dt, int interp,
                      int backtrace, const void *gphi, void *gphi0, void *gvel, cudaStream_t st);

// Exclusive scan of n ints (in may alias out); *total = the sum, FLAG_CAPACITY
// raised in flags when it exceeds cap.  partial: scan_partial_ints(n) ints.
size_t scan_partial_ints(long long n);
int launch_scan_exclusive(const int *in, int n, int *out, int *partial, int *total, int cap, int *flags,
                          cudaStream_t st);

size_t irregular_scratch_bytes(int nband);
int launch_irregular(const dcell::Geom &g, int dtype, const void *phi, const int *band, int nband, int with_surface,
                     dcell_irregular_node *nodes, int cap, int *count, void *scratch, int *flags, cudaStream_t st);
int launch_max_velocity(const dcell::Geom &g, int dtype, const void *vel, const dcell_irregular_node *nodes,
                        const int *count, int cap, double *out, cudaStream_t st);
// Allocation-free irregular-node pass: scratch in a static device array.
constexpr int kNoAllocMaxBand = 1 << 20;
constexpr int kNoAllocScratchInts = kNoAllocMaxBand + 1 + (kNoAllocMaxBand + 1023) / 1024 + 1;
constexpr int kNoAllocMaxDevices = 64;
int launch_irregular_noalloc(const dcell::Geom &g, int dtype, const void *phi, const int *band, int nband,
                             int with_surface, dcell_irregular_node *nodes, int cap, int *count, int *flags,
                             cudaStream_t st);
int launch_velocity_box(const dcell::Geom &g, int dtype, const void *global, const int gdims[3], int gdof, int first,
                        void *vel, cudaStream_t st);
int launch_velocity_boxes(const dcell_box *boxes, int nboxes, int dim, int dtype, const void *global,
                          const int gdims[3], int gdof, int first, long long max_points, void *vel, cudaStream_t st);
// max |v[comp]| over n points of a dof-component FP32 field, atomicMax'ed
// into *out as FP32 bits (initialise *out to 0)
// range: updated global index range [xs, xe, ys, ye, zs, ze) (2D: zs = 0, ze = 1)
int launch_advect_mac(const dcell::Geom &g, int dtype, const void *phi, const void *u, const void *v, const void *w,
                      double dt, const int range[6], void *out, cudaStream_t st);
int launch_max_abs_component(const float *v, long long n, int dof, int comp, int *out, cudaStream_t st);
size_t reinit_scratch_bytes(long long n, int dtype);
int launch_reinit(const dcell::Geom &g, int dtype, void *phi, const dcell_irregular_node *nodes, int nnodes, double bw,
                  double bucket, int *band, int cap, int *count, void *scratch, int *flags, cudaStream_t st);
size_t volume_scratch_bytes();
int launch_volume(const dcell::Geom &g, int dtype, const void *phi, double eps, double *out, double *partial,
                  cudaStream_t st);

int launch_convert(const void *src, int src_dtype, void *dst, int dst_dtype, long long n, cudaStream_t st);
int launch_gather_band(const dcell::Geom &g, int dtype, const void *phi, const int *band, int nband, void *out,
                       cudaStream_t st);

// particle level set (pls.cu)
int launch_pls_advect(const dcell::Geom &g, int dtype, const void *vel, void *parts, long long n, double dt,
                      int *flags, cudaStream_t st);
size_t pls_correct_scratch_bytes(long long npts, int dtype);
int launch_pls_correct(const dcell::Geom &g, int dtype, void *phi, const int *band, long long nband,
                       const void *parts, long long n, void *scratch, int *flags, cudaStream_t st);
int launch_pls_adjust(const dcell::Geom &g, int dtype, const void *phi, void *parts, long long n,
                      const dcell_pls_params &prm, int *flags, cudaStream_t st);
size_t pls_scratch_bytes(long long npts, long long nband, long long n);
int launch_pls_seed(const dcell::Geom &g, int dtype, const void *phi, const int *band, long long nband,
                    const dcell_pls_params &prm, unsigned long long *rng, void *parts, long long cap, long long *count,
                    void *scratch, int *flags, cudaStream_t st);
int launch_pls_reseed(const dcell::Geom &g, int dtype, const void *phi, const int *band, long long nband,
                      const dcell_pls_params &prm, unsigned long long *rng, void *parts, long long n, long long cap,
                      long long *count, void *scratch, int *flags, cudaStream_t st);
