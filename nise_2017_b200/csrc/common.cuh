// Device-side helpers shared by the engine's kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define NISE_HD __host__ __device__ __forceinline__

// Packed upper-triangle index of (a,b), row-major over a <= b
// (Sindex, NISE_subs.h:54-65).
NISE_HD int sindex(int a, int b, int n) {
    if (a > b) return a + b * ((n << 1) - b - 1) / 2;
    return b + a * ((n << 1) - a - 1) / 2;
}

template <typename R> struct Vec2;
template <> struct Vec2<float> { typedef float2 T; };
template <> struct Vec2<double> { typedef double2 T; };

// Arithmetic policy.  Exact<float> issues every single-precision multiply,
// add and subtract as a separately rounded operation (no contraction into
// fused multiply-add), which is how the reference's C code is evaluated on
// x86-64; the double policy lets the compiler fuse.
template <typename R> struct Ar;
template <> struct Ar<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};
template <> struct Ar<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return a * b; }
    static __device__ __forceinline__ double add(double a, double b) { return a + b; }
    static __device__ __forceinline__ double sub(double a, double b) { return a - b; }
};

#include "devtypes.h"

// Shifted diagonal element of frame t, before SingleShift.
__device__ __forceinline__ float traj_diag_raw(const DevTraj &T, long t, int i) {
    const float *rec = T.energy + t * T.e_words + 1;
    float h = T.full ? rec[sindex(i, i, T.n)] : rec[i];
    return __fsub_rn(h, T.shifte);
}

// Shifted diagonal with SingleShift applied (read_Hamiltonian,
// read_trajectory.c:73-87 -> apply_singleshift, hamshift.c:59-66).  The
// reference applies the file's entries in order; a site's own entries are
// looked up through shift_ptr and applied in the same order, so a site named
// twice gets the same two roundings.
__device__ __forceinline__ float traj_diag(const DevTraj &T, long t, int i, bool singleshift) {
    float h = traj_diag_raw(T, t, i);
    if (singleshift)
        for (int e = T.shift_ptr[i]; e < T.shift_ptr[i + 1]; e++)
            h = __fadd_rn(__fmul_rn(h, T.shift_ab[2 * e]), T.shift_ab[2 * e + 1]);
    return h;
}

// Off-diagonal element (a < b) of frame t after the read cut
// (read_trajectory.c:305-311: |J| < cut -> 0).
__device__ __forceinline__ float traj_coupling(const DevTraj &T, long t, int a, int b) {
    int idx = sindex(a, b, T.n);
    float j = T.full ? T.energy[t * T.e_words + 1 + idx] : T.hc[idx];
    return fabsf(j) < T.cut ? 0.0f : j;
}

// Dipole component x of site i at frame t (read_mue :357-377 or the static
// dipoles of HamiltonianType Coupling, read_coupling :47-70).
__device__ __forceinline__ float traj_mu(const DevTraj &T, long t, int x, int i) {
    if (T.mu_static) return T.mu_static[x * T.n + i];
    return T.dipole[t * T.d_words + 1 + x * T.n + i];
}

