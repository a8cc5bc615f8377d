// Frame builder for couplings computed on the fly (HamiltonianType
// TransitionDipole / ExtendedDipole, read_trajectory.c:180-303).
//
// The reference recomputes every coupling of a frame each time it reads the
// frame, once per vector and step.  Here one kernel builds every frame's Full
// record image in HBM once: the diagonal from the Hamiltonian file's
// diagonal records, the couplings from the positions, the transition dipoles
// and the periodic box of the frame.  The propagators then read these records
// like a HamiltonianType Full trajectory (the Couplingcut is applied when a
// coupling is read, as read_He does after computing them).
//
// The arithmetic follows the reference's float expressions operation by
// operation (no fused multiply-add); its sqrt() and 1.0/x are evaluated in
// double and rounded to float, as the C calls are.
#include "common.cuh"
#include "engine.h"

namespace {

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

// pbc1 (NISE_subs.c:641-648)
__device__ __forceinline__ float pbc1(float r, int x, const float *box) {
    if (box[0] > 0.0f) {
        if (r > __fdiv_rn(box[x], 2.0f)) r = fs(r, box[x]);
        if (r < __fdiv_rn(-box[x], 2.0f)) r = fa(r, box[x]);
    }
    return r;
}

// float(sqrt(double(x))) and float(1.0 / double(x))
__device__ __forceinline__ float csqrt(float x) { return (float)__dsqrt_rn((double)x); }
__device__ __forceinline__ float cinv(float x) { return (float)__ddiv_rn(1.0, (double)x); }

__device__ __forceinline__ float norm2(float x, float y, float z) { return fa(fa(fm(x, x), fm(y, y)), fm(z, z)); }

// One thread per (frame, site i): the diagonal element and the couplings (i, j > i).
__global__ void k_onfly(OnflyJob J, float *out) {
    const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (g >= J.frames * J.n) return;
    const long t = g / J.n;
    const int n = J.n, i = (int)(g % J.n);
    float *rec = out + t * J.full_words;
    const float *diag = J.diag + t * (1 + n);
    if (i == 0) {
        ((int *)rec)[0] = ((const int *)diag)[0];  // the record's int32 tag
        for (long w = 1 + (long)n * (n + 1) / 2; w < J.full_words; w++) rec[w] = 0.f;
    }
    rec[1 + sindex(i, i, n)] = diag[1 + i];
    float box[3] = {0.f, 0.f, 0.f};
    if (J.pbc) {
        const float *b = J.pbc + t * 4 + 1;
        box[0] = b[0];
        box[1] = b[1];
        box[2] = b[2];
    }
    const long prec = J.dip_words;  // position records have the dipole records' layout (read_mue)
    const float *R = J.pos + (J.edc ? 2 * t : t) * prec + 1;
    const float *R2 = J.edc ? R + prec : R;
    const float *mu = J.dip + t * J.dip_words + 1;
    const float A = 5034.11861687f;
    const float m1x = mu[i], m1y = mu[n + i], m1z = mu[2 * n + i];
    if (!J.edc) {
        for (int j = i + 1; j < n; j++) {
            float Rx = pbc1(fs(R[i], R[j]), 0, box);
            float Ry = pbc1(fs(R[n + i], R[n + j]), 1, box);
            float Rz = pbc1(fs(R[2 * n + i], R[2 * n + j]), 2, box);
            float m2x = mu[j], m2y = mu[n + j], m2z = mu[2 * n + j];
            float dist = csqrt(norm2(Rx, Ry, Rz));
            float idist = cinv(dist);
            float idist3 = fm(fm(idist, idist), idist);
            float f1 = fa(fa(fm(m1x, m2x), fm(m1y, m2y)), fm(m1z, m2z));
            float d1 = fa(fa(fm(m1x, Rx), fm(m1y, Ry)), fm(m1z, Rz));
            float d2 = fa(fa(fm(m2x, Rx), fm(m2y, Ry)), fm(m2z, Rz));
            float f2 = fm(fm(fm(fm(-3.0f, d1), d2), idist), idist);
            rec[1 + sindex(i, j, n)] = fm(fm(A, fa(f1, f2)), idist3);
        }
    } else {
        float Rx = pbc1(fs(R2[i], R[i]), 0, box);
        float Ry = pbc1(fs(R2[n + i], R[n + i]), 1, box);
        float Rz = pbc1(fs(R2[2 * n + i], R[2 * n + i]), 2, box);
        float dist = csqrt(norm2(Rx, Ry, Rz));
        const double m1 = __dsqrt_rn((double)norm2(m1x, m1y, m1z));
        const float q1 = (float)__ddiv_rn(m1, (double)dist);
        for (int j = i + 1; j < n; j++) {
            Rx = pbc1(fs(R2[j], R[j]), 0, box);
            Ry = pbc1(fs(R2[n + j], R[n + j]), 1, box);
            Rz = pbc1(fs(R2[2 * n + j], R[2 * n + j]), 2, box);
            dist = csqrt(norm2(Rx, Ry, Rz));
            // the reference forms q2 from the first site's dipole (read_trajectory.c:246)
            const float q2 = (float)__ddiv_rn(m1, (double)dist);
            float Jc;
            Rx = pbc1(fs(R[i], R[j]), 0, box);
            Ry = pbc1(fs(R[n + i], R[n + j]), 1, box);
            Rz = pbc1(fs(R[2 * n + i], R[2 * n + j]), 2, box);
            Jc = cinv(csqrt(norm2(Rx, Ry, Rz)));
            Rx = pbc1(fs(R[i], R2[j]), 0, box);
            Ry = pbc1(fs(R[n + i], R2[n + j]), 1, box);
            Rz = pbc1(fs(R[2 * n + i], R2[2 * n + j]), 2, box);
            Jc = fs(Jc, cinv(csqrt(norm2(Rx, Ry, Rz))));
            Rx = pbc1(fs(R2[i], R[j]), 0, box);
            Ry = pbc1(fs(R2[n + i], R[n + j]), 1, box);
            Rz = pbc1(fs(R2[2 * n + i], R[2 * n + j]), 2, box);
            Jc = fs(Jc, cinv(csqrt(norm2(Rx, Ry, Rz))));
            Rx = pbc1(fs(R2[i], R2[j]), 0, box);
            Ry = pbc1(fs(R2[n + i], R2[n + j]), 1, box);
            Rz = pbc1(fs(R2[2 * n + i], R2[2 * n + j]), 2, box);
            Jc = fa(Jc, cinv(csqrt(norm2(Rx, Ry, Rz))));
            rec[1 + sindex(i, j, n)] = fm(fm(fm(A, q1), q2), Jc);
        }
    }
}

}  // namespace

int launch_onfly(const OnflyJob &J, float *out, cudaStream_t s) {
    long tot = J.frames * J.n;
    if (tot <= 0) return 0;
    k_onfly<<<(unsigned)((tot + 127) / 128), 128, 0, s>>>(J, out);
    return (int)cudaGetLastError();
}
