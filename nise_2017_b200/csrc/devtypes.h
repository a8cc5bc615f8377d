// Plain data types shared by host code (api.cpp) and device code.
#pragma once
#include <vector_types.h>

// Trajectory records as the reference reads them (read_trajectory.c):
// every record is an int32 tag followed by float32 data, addressed here in
// 4-byte words so the tag is word 0.
struct DevTraj {
    const float *energy;     // energy record image
    long e_words;            // words per energy record
    long e_frames;
    int full;                // 1: packed N(N+1)/2 (+doubles) frames; 0: N diagonal values
    const float *dipole;     // dipole record image (per-frame dipoles)
    long d_words;
    long d_frames;
    const float *mu_static;  // [3][N] for HamiltonianType Coupling (else nullptr)
    const float *hc;         // packed coupling frame (HamiltonianType Coupling), cut applied
    const float *anh;        // anharmonicity records (N per frame) or nullptr
    long a_frames;
    const float *over;       // overtone dipole records (3N per frame) or nullptr
    long o_frames;
    const int *shift_ptr;    // SingleShift entries of site i: shift_ab[2e], e in [shift_ptr[i], shift_ptr[i+1])
    const float *shift_ab;   // (a, b) pairs, grouped by site in file order
    int nshift;
    int n;                   // singles
    float shifte;            // (min1 + max1) / 2
    float cut;               // Couplingcut
};

// Coefficient tables of one singles propagation scheme over the frames
// [f0, f0 + nf) of a job (built by nise_singles_tables): the Trotter half
// phases U[t][n] and rotations rot[t][K] (or [K] for static couplings), the
// RK4 Hamiltonian entries, or the eigen route's one-step propagators
// Ud[t][n][n].  Device code reads them through singles_step (schemes.cuh).
struct SinglesTab {
    int n, ts, prop;          // singles, Trotter sub-steps, NISE_PROP_*
    long f0;                  // first frame of the tables
    const int2 *pairs;        // Trotter pattern (a < b, lexicographic)
    int K;
    const int4 *segs;         // the pattern in segments of one first site a and one warp of
    int nsegs;                // second sites (b >> 5): (a, first, end, b >> 5)
    const void *U, *rot;      // Trotter tables
    int rot_static;
    const int2 *ent;          // RK4 entries (a <= b)
    int Kr;
    const void *rkval;        // RK4 values [t][Kr]
    const void *Ud;           // Sparse/Diagonal: propagators U[t][n][n] (truncated by Threshold)
};
