/* scenes.h -- seeded synthetic workloads (see scenes.c for the definitions). */
#ifndef QUARRY_B200_SCENES_H
#define QUARRY_B200_SCENES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

double qs_det_sin(double x);
double qs_det_cos(double x);
double qs_det_log(double x);
double qs_det_exp(double x);

int64_t qs_cfg_terrain(int grid, uint64_t seed, float* tris9);
void qs_cfg_down_rays(int count, float x0, float x1, float y0, float y1, float z, uint64_t seed,
                      float* rays8);
void qs_cfg_cosine_rays(int count, float x0, float x1, float y0, float y1, float z,
                        uint64_t seed, float* rays8);
void qs_cfg_uniform_points(int count, const float* lo3, const float* hi3, uint64_t seed,
                           uint64_t stream, float* pts3);
int64_t qs_cfg_city(int buildings, uint64_t seed, float* tris9, float* max_height);
void qs_cfg_points(int kind, int count, uint64_t seed, float* pts3);
void qs_cfg_coherent_motion(const float* pts3, int count, int dirty, float sigma, uint64_t seed,
                            float* out3, int32_t* ids);
void qs_cfg_gaussians(int count, float smin, float smax, uint64_t seed, float* g10);
int qs_log_uniform_int(uint64_t seed, uint64_t stream, int lo, int hi);

int64_t qs_demo_mesh(int kind, int grid, int random_tris, uint64_t seed, int buildings,
                     float* tris9);
void qs_demo_gaussians(int kind, int count, uint64_t seed, float* g10);

#ifdef __cplusplus
}
#endif

#endif
