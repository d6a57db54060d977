// ref_shim.h -- TEST INFRASTRUCTURE.  Force-included (nvcc -include) when oracle/build_ref.py
// compiles the reference's own motion_stereo/*.cu sources, unmodified and where they lie, into
// oracle/_ref/ for pinning the oracle.  Two things stop those sources from building on CUDA 12:
//
//  1. Texture references (`texture<float, cudaTextureType2D, ...>`, tex2D(ref, x, y),
//     cudaBindTexture2D, cudaUnbindTexture) were removed.  Below, `texture` becomes a small
//     host struct that records the addressing/filter settings the reference assigns, tex2D on a
//     named reference becomes a fetch through a texture object held in a __device__ variable of
//     the same name stem, and cudaBindTexture2D creates that object with the recorded settings.
//  2. The image shape is compile-time (parameters.h).  Defining the header's include guard here
//     and declaring the same names lets one build the reference at a small test shape
//     (PM_REF_W x PM_REF_H x PM_REF_D); the mutable parameters keep their definitions in the
//     reference's parameters.cpp.
#pragma once
#include <cuda_runtime.h>
#include <texture_fetch_functions.h>
#include <cstring>

#include "ref_params.h"

// ---- texture references on top of texture objects ---------------------------------------
template <class T, int Dim, enum cudaTextureReadMode Mode>
struct pm_ref_texture {
    int addressMode[3] = {0, 0, 0};
    int filterMode = 0;
    bool normalized = false;
    cudaTextureObject_t obj = 0;
    cudaTextureObject_t* slot = nullptr;   // host shadow of the __device__ object variable
};
#define texture pm_ref_texture

__device__ cudaTextureObject_t pm_ref_obj_tex2Dleft;
__device__ cudaTextureObject_t pm_ref_obj_tex2Dright;
__device__ __forceinline__ float pm_ref_fetch_tex2Dleft(float x, float y) {
    return tex2D<float>(pm_ref_obj_tex2Dleft, x, y);
}
__device__ __forceinline__ float pm_ref_fetch_tex2Dright(float x, float y) {
    return tex2D<float>(pm_ref_obj_tex2Dright, x, y);
}
#define tex2D(t, x, y) pm_ref_fetch_##t(x, y)

template <class T, int Dim, enum cudaTextureReadMode Mode>
cudaError_t cudaUnbindTexture(pm_ref_texture<T, Dim, Mode>& t) {
    if (t.obj) cudaDestroyTextureObject(t.obj);
    t.obj = 0;
    return cudaSuccess;
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
cudaError_t cudaBindTexture2D(size_t* offset, pm_ref_texture<T, Dim, Mode>& t, const void* ptr,
                              const cudaChannelFormatDesc& desc, size_t w, size_t h, size_t pitch) {
    if (offset) *offset = 0;
    if (!t.slot) return cudaErrorInvalidValue;
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof rd);
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = const_cast<void*>(ptr);
    rd.res.pitch2D.desc = desc;
    rd.res.pitch2D.width = w;
    rd.res.pitch2D.height = h;
    rd.res.pitch2D.pitchInBytes = pitch;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof td);
    for (int i = 0; i < 3; ++i) td.addressMode[i] = (cudaTextureAddressMode)t.addressMode[i];
    td.filterMode = (cudaTextureFilterMode)t.filterMode;
    td.readMode = Mode;
    td.normalizedCoords = t.normalized ? 1 : 0;
    if (t.obj) cudaDestroyTextureObject(t.obj);
    cudaError_t e = cudaCreateTextureObject(&t.obj, &rd, &td, nullptr);
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(*t.slot, &t.obj, sizeof(t.obj));
}
