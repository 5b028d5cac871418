// Host-side entry points shared between the library's translation units (not
// public ABI).
#pragma once

#include "../../include/lcbinint_b200.h"

namespace lcbi {

// Finite-source magnification of host points through LensModel's decision
// (src/lcbinint/model/lens_model.cpp:200-226): each point's point-source value
// and image count come from binary_images on the device (binary_mag0 for
// rho == 0), its images seed the inverse ray (LCBI_FS_SEED_HINTS), and the
// value is exact for the hexadecapole (LCBI_FS_PS_EXACT).  points[i].flags and
// point_source_magnification are ignored; points[i].model is assigned here.
// Points are processed in chunks that bound the caustic samples held on the
// device, so per-point separations (lens orbital motion) need no more memory
// than a chunk's.  results, a_ps, image_count and levels (optional: the
// adaptive refinement level of each point) have n entries.
int binary_mag_images(lcbi_gpu_context* ctx, const lcbi_fs_settings* settings, int n_settings,
                      const lcbi_fs_point* points, long long n, lcbi_fs_result* results, double* a_ps,
                      int32_t* image_count, int32_t* levels);

} // namespace lcbi
