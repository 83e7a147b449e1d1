// Host-side helpers shared by the C-ABI entry points: argument checks, the
// per-frame camera block, launch status.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/dgmr_b200.h"
#include "dgmr_device_math.cuh"

namespace dgmr {

inline dgmr_status check_scene(const dgmr_scene* scene, const dgmr_camera* camera, int required_dtype)
{
    if (!scene || !camera)
        return DGMR_ERR_BAD_ARG;
    if (scene->n_gaussians < 0 || camera->width <= 0 || camera->height <= 0 || camera->width > 65536 || camera->height > 65536)
        return DGMR_ERR_BAD_ARG;
    if (scene->sh_stride < 1 || scene->sh_stride > 16 || scene->sh_degree < 0 || scene->sh_degree > 3)
        return DGMR_ERR_BAD_ARG;
    if (required_dtype >= 0 && scene->dtype != required_dtype)
        return DGMR_ERR_BAD_ARG;
    if (scene->dtype != DGMR_F32 && scene->dtype != DGMR_F64)
        return DGMR_ERR_BAD_ARG;
    if (scene->n_gaussians > 0
        && (!scene->centroids || !scene->sh || !scene->weights || !scene->scales || !scene->rotations))
        return DGMR_ERR_BAD_ARG;
    if (scene->formulation < DGMR_FORMULATION_DEFAULT || scene->formulation > DGMR_FORMULATION_OLS)
        return DGMR_ERR_BAD_ARG;
    return DGMR_OK;
}

// the scene's formulation, or the renderer's reference default
inline Formulation scene_formulation(const dgmr_scene* scene, Formulation renderer_default)
{
    if (!scene || scene->formulation == DGMR_FORMULATION_DEFAULT)
        return renderer_default;
    return Formulation(scene->formulation - 1);
}

// glm::inverse of a 4x4 (glm layout) by cofactors, evaluated in double
inline void inverse4_glm(const double* m, double* inv_out)
{
    double inv[16];
    inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
    inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
    inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
    inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
    inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
    inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
    inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
    inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
    inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
    inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
    inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
    inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
    inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
    inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
    inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
    inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
    const double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
    for (int i = 0; i < 16; ++i)
        inv_out[i] = inv[i] / det;
}

// Per-frame camera block in the kernel's precision.  Values are first
// rounded to T, then combined in T, exactly as the reference does with
// its typed ForwardData (vol_marcher_forward.cu:53-58).
template <class T>
inline CameraT<T> make_camera(const dgmr_camera& c)
{
    CameraT<T> k;
    double inv[16], proj_t[16];
    for (int i = 0; i < 16; ++i) {
        k.view[i] = T(c.view[i]);
        k.proj[i] = T(c.proj[i]);
        proj_t[i] = double(k.proj[i]);
    }
    inverse4_glm(proj_t, inv);
    for (int i = 0; i < 16; ++i)
        k.inv_proj[i] = T(inv[i]);
    for (int i = 0; i < 3; ++i) {
        k.campos[i] = T(c.campos[i]);
        k.bg[i] = T(c.background[i]);
    }
    k.tan_fovx = T(c.tan_fovx);
    k.tan_fovy = T(c.tan_fovy);
    k.W = unsigned(c.width);
    k.H = unsigned(c.height);
    k.focal_y = T(float(k.H)) / (T(2.0f) * k.tan_fovy);
    k.focal_x = T(float(k.W)) / (T(2.0f) * k.tan_fovx);
    k.cov_scale_multiplier = T(c.cov_scale_multiplier);
    k.gx = (k.W + kTile - 1) / kTile;
    k.gy = (k.H + kTile - 1) / kTile;
    return k;
}

inline int num_sms()
{
    static int cached = 0;
    if (cached == 0) {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached = n > 0 ? n : 148;
    }
    return cached;
}

inline dgmr_status launch_status()
{
    return cudaGetLastError() == cudaSuccess ? DGMR_OK : DGMR_ERR_CUDA;
}

} // namespace dgmr
