// Per-event spin-orbit amplitude tensors on the device (init time).
//
// For every event and every angular group (decay chain x intermediate J^P)
// this builds the two-body covariant amplitude tensor of each decay vertex,
//   T[s][s1][s2] = 10 q^L / sqrt(2J+1) <j1 s1 j2 s2|S s1+s2> <S s1+s2, L m|J s> Y_L^m(theta, -phi)
//                  followed by the daughters' Wigner rotations,
// (the reference's pwa_amp, src/Amplitude.cu:237-644), contracts the vertex
// tensors along the chain (src/AmpGen.cu:1034-1219) and stores the result as
// SoA planes [plane][pol][event]. Clebsch-Gordan products and Wigner small-d
// sum coefficients are tabulated on the host; the device evaluates only the
// event-dependent parts (frames, Legendre functions, phases, rotations).
#pragma once

#include <cuComplex.h>

#define AG_MAXP 16     // particles per group
#define AG_MAXN 8      // decay vertices per chain
#define AG_MAXD 7      // 2J+1 (J <= 3)
#define AG_MAXT 64     // complex elements of any intermediate tensor

struct AgNodeVar {  // one (S, L) choice of a vertex
    int S, L;
    int cg_off;     // offset of dj*dj1*dj2 doubles: CG1*CG2/sqrt(dj), 0 where forbidden
};

struct AgNode {
    int mother, d1, d2;
    int dj, dj1, dj2;
    int var_off, nvar;
};

struct AgGroup {
    int np, nfin, nnodes, nsl, npol, tensor_size;
    int plane0;          // first output plane of this group
    int input_slot[AG_MAXP];
    int sum_a[AG_MAXP], sum_b[AG_MAXP];
    int build_order[AG_MAXP];
    AgNode nodes[AG_MAXN];
    const int* sl_var;   // [nsl][nnodes] variant index per vertex
    const int* pol_map;  // [npol] or nullptr
    int nkin;            // kinematic slots filled by this group
    const int* kin;      // [nkin][5]: type, a, b, c, out slot
};

struct AgTables {
    const AgNodeVar* vars;
    const double* cg;       // CG products
    const double* ylm_norm; // [l][|m|] sqrt((2l+1)/(4 pi) (l-|m|)!/(l+|m|)!) , l < AG_MAXD
    const double* dcoef;    // Wigner small-d sum coefficients (see dsmall)
    const int* doff;        // [dim][m1][m2] -> offset into dcoef (count first)
};

// kinematic slot types
#define AG_K_MASS 0      // M() of particle a
#define AG_K_Q 1         // breakup(M(a), M(b), M(c)), 0 below threshold
#define AG_K_QRAW 2      // sqrt((m^2-(m1+m2)^2)(m^2-(m1-m2)^2))/2/m without clamp
#define AG_K_P 3         // |p| of particle a
#define AG_K_E 4         // E of particle a
#define AG_K_CT 5        // p_z/|p| (0 if |p| = 0)
#define AG_K_PHI 6       // atan2(p_y, p_x)
