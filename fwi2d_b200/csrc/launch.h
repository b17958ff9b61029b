// Host entry points of the kernels in kernels.cu.
#pragma once
#include "engine.h"

namespace fwi2d {

enum StepFlagBits { STEP_STORE = 1, STEP_EXTRACT = 2, STEP_AMAX = 4, STEP_GRAD = 8 };

void upload_sbp_tables(const float *b1, const float *b2, const float *c2, const float *c1, const float *sc,
                       const float *hc);

int elastic_tile_count();
void elastic_tile_shape(int i, int *tz, int *tx);
// the x-band windows (32 x 8, full height) of framed and marching plans:
// split = true takes the band kernel that updates the two components of a
// cell in two warps (xband.cuh), split = false the tile kernel's general path
void launch_elastic_xband(bool vti, bool split, const ShotDev *shots, const TileRef *tiles, int ntiles,
                          const ModelDev &M, const StepConst &C, int it, int flags, float dtg, cudaStream_t st);
void launch_elastic_step(int shape, bool vti, const ShotDev *shots, const TileRef *tiles, int ntiles,
                         const ModelDev &M, const StepConst &C, int it, int flags, float dtg, cudaStream_t st,
                         bool core = false);
// x-marching kernel for the cells clear of all four boundary bands; nth
// threads per unit (one z cell each), a width march_threads_ok accepts
bool march_threads_ok(int nth);
void launch_elastic_march(bool vti, const ShotDev *shots, const MarchRef *units, int nunits, int nth,
                          const ModelDev &M, const StepConst &C, int it, int flags, float dtg, cudaStream_t st);
// top / bottom band kernel (rows clear of the x bands), zband_rows(split)
// rows per unit; split as for the x bands
int zband_rows(bool split);
void launch_elastic_zband(bool vti, bool split, const BandRef *units, int nunits, const ShotDev *shots,
                          const ModelDev &M, const StepConst &C, int it, int flags, float dtg, cudaStream_t st);
void launch_init_state(const ShotDev *shots, int nshots, const InitCell *cells, const int *off, const int *idx,
                       cudaStream_t st);
// Receivers of the last sample and its snapshot (t_store < 0), or only the
// snapshot of time sample t_store (flags = STEP_STORE).
void launch_finalize(const ShotDev *shots, int nshots, const StepConst &C, int ncomp, int flags, cudaStream_t st,
                     int t_store = -1);
// Copy both field buffers of every shot to / from checkpoint k (ShotDev::ckpt).
void launch_checkpoint(const ShotDev *shots, int nshots, int ncomp, int k, bool restore, cudaStream_t st);

// acoustic kernel (acoustic.cuh): tile shapes 2 and 3 only
bool acoustic_shape_ok(int shape);
void launch_acoustic_step(int shape, const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                          const StepConst &C, int it, int flags, float dtg, cudaStream_t st);
void launch_ae_fluid_step(int shape, const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                          const StepConst &C, int it, int flags, cudaStream_t st);
void launch_ae_elastic_step(int shape, const ShotDev *shots, const TileRef *tiles, int ntiles, const ModelDev &M,
                            const StepConst &C, int it, int flags, float dtg, cudaStream_t st);
void launch_ae_couple(const ShotDev *elastic, const ShotDev *fluid, int nshots, int nx_max, const ModelDev &M,
                      const StepConst &C, int it, int flags, float dtg, float Kw, float val0, int sign, cudaStream_t st);
void launch_acoustic_final_grad(const ShotDev *shots, int nshots, const ModelDev &M, const StepConst &C, float dtg,
                                cudaStream_t st);
// Move the marching kernel's timeout flag (the row + 1 where a bounded wait
// gave up, 0 if none) into *status unless it already holds one, and clear it.
void launch_take_timeout(int *status, cudaStream_t st);

// layout helpers (engine.cu)
void launch_to_time_major(const float *in, float *out, int rows, int nt, cudaStream_t st);
void launch_from_time_major(const float *in, float *out, int rows, int nt, cudaStream_t st);
void launch_add_subgrid(float *full, const float *part, int ncomp, int x0, int nx, int ldz, long long full_comp,
                        cudaStream_t st);

}  // namespace fwi2d
