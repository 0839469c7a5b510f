// Lattice constants shared by host and device code.
//
// Direction order, weights and the MRT moment basis follow the reference
// (lbm_project/d2q9_model/lbm_d2q9.h:53-92, lbm_project/d3q19_model/lbm_d3q19.h:18-167)
// so that populations exchanged through the C ABI use the reference's indexing.
// Tables are constexpr functions so device code can index them with loop
// variables that the compiler folds after unrolling.
#pragma once
#include <cstdint>

#ifndef ZL_HD
#define ZL_HD __host__ __device__ __forceinline__
#endif

namespace zl {

struct D2Q9 {
    static constexpr int kDims = 2;
    static constexpr int kQ = 9;
    static constexpr int kFaceQ = 3;
};
struct D3Q19 {
    static constexpr int kDims = 3;
    static constexpr int kQ = 19;
    static constexpr int kFaceQ = 5;
};

template <class L> struct Tables;

template <> struct Tables<D2Q9> {
    ZL_HD static constexpr int cx(int q) {
        constexpr int t[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
        return t[q];
    }
    ZL_HD static constexpr int cy(int q) {
        constexpr int t[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
        return t[q];
    }
    ZL_HD static constexpr int cz(int) { return 0; }
    ZL_HD static constexpr int opp(int q) {
        constexpr int t[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
        return t[q];
    }
    ZL_HD static constexpr double w(int q) {
        return q == 0 ? 4. / 9. : (q < 5 ? 1. / 9. : 1. / 36.);
    }
    // MRT basis (Lallemand & Luo 2000), rows are moments
    ZL_HD static constexpr int M(int k, int j) {
        constexpr int t[9][9] = {
            {1, 1, 1, 1, 1, 1, 1, 1, 1},      {-4, -1, -1, -1, -1, 2, 2, 2, 2},
            {4, -2, -2, -2, -2, 1, 1, 1, 1},  {0, 1, 0, -1, 0, 1, -1, -1, 1},
            {0, -2, 0, 2, 0, 1, -1, -1, 1},   {0, 0, 1, 0, -1, 1, 1, -1, -1},
            {0, 0, -2, 0, 2, 1, 1, -1, -1},   {0, 1, -1, 1, -1, 0, 0, 0, 0},
            {0, 0, 0, 0, 0, 1, -1, 1, -1}};
        return t[k][j];
    }
    // relaxation rates of the moments; -1 marks the shear moments that take 1/tau
    ZL_HD static constexpr double s(int k) {
        constexpr double t[9] = {0., 1.4, 1.4, 0., 1.2, 0., 1.2, -1., -1.};
        return t[k];
    }
};

template <> struct Tables<D3Q19> {
    ZL_HD static constexpr int cx(int q) {
        constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
        return t[q];
    }
    ZL_HD static constexpr int cy(int q) {
        constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
        return t[q];
    }
    ZL_HD static constexpr int cz(int q) {
        constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
        return t[q];
    }
    ZL_HD static constexpr int opp(int q) {
        constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
        return t[q];
    }
    ZL_HD static constexpr double w(int q) {
        return q == 0 ? 1. / 3. : (q < 7 ? 1. / 18. : 1. / 36.);
    }
    // MRT basis (d'Humieres et al. 2002), rows are moments
    ZL_HD static constexpr int M(int k, int j) {
        constexpr int t[19][19] = {
            {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
            {-30, -11, -11, -11, -11, -11, -11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8},
            {12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
            {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
            {0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
            {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1},
            {0, 0, 0, -4, 4, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1},
            {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
            {0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1},
            {0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
            {0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
            {0, 0, 0, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
            {0, 0, 0, -2, -2, 2, 2, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
            {0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 0, 0, 0, 0},
            {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1},
            {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0},
            {0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0},
            {0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, 1, -1, 1, -1},
            {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, -1, -1, 1, 1}};
        return t[k][j];
    }
    ZL_HD static constexpr double s(int k) {
        constexpr double t[19] = {0., 1.5, 1.4, 0., 1.2, 0., 1.2, 0., 1.2, -1.,
                                  1.4, -1., 1.4, -1., -1., -1., 1.98, 1.98, 1.98};
        return t[k];
    }
};

// Squared norm of MRT row k (the basis is orthogonal: M^-1 = M^T diag(1 / |M_k|^2)).
template <class L>
ZL_HD constexpr int row_norm2(int k) {
    int acc = 0;
    for (int j = 0; j < L::kQ; ++j) acc += Tables<L>::M(k, j) * Tables<L>::M(k, j);
    return acc;
}

// Face slots in the reference's naming: xmin, xmax, ymin, ymax, zmin, zmax.
enum Face : int { kXMin = 0, kXMax = 1, kYMin = 2, kYMax = 3, kZMin = 4, kZMax = 5 };

// Whether direction q enters the domain through face f (c_axis > 0 on a min face, < 0 on a max face);
// these are the reference's per-face index lists (boundary_conditions/lbm_boundary_conditions.cpp:102-156).
template <class L>
ZL_HD constexpr bool enters_through(int q, int face) {
    const int axis = face >> 1;
    const int c = axis == 0 ? Tables<L>::cx(q) : (axis == 1 ? Tables<L>::cy(q) : Tables<L>::cz(q));
    return (face & 1) ? (c < 0) : (c > 0);
}

// Source direction of the bounce-back for a population q entering through `face`: the
// reference pairs the n-th entry of its per-axis "positive" and "negative" index lists
// (d2q9_model/lbm_d2q9.h:62-67, d3q19_model/lbm_d3q19.h:86-95, used by
// boundary_conditions/lbm_bounce_back.cpp:28-91).  For D3Q19 every pair is an opposite pair.
// For D2Q9 the x lists are {1, 8, 5} / {3, 7, 6}: the diagonals of an x wall are reflected
// specularly (8 <- 7, 5 <- 6) while y walls reflect them back (5 <- 7, 6 <- 8).
template <class L>
ZL_HD constexpr int bb_source(int q, int face) {
    if constexpr (L::kQ == 9) {
        if ((face >> 1) == 0) {
            constexpr int xmin[9] = {0, 3, 0, 0, 0, 6, 0, 0, 7};  // 1<-3, 5<-6, 8<-7
            constexpr int xmax[9] = {0, 0, 0, 1, 0, 0, 5, 8, 0};  // 3<-1, 6<-5, 7<-8
            return (face & 1) ? xmax[q] : xmin[q];
        }
        return Tables<L>::opp(q);
    } else {
        return Tables<L>::opp(q);
    }
}

}  // namespace zl
