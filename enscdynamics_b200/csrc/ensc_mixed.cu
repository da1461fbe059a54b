// Mixed-precision stepper kernels: the element pass (kinematics, Jaumann /
// J2 stress, hourglass, bulk viscosity) and the force gather run in FP32;
// nodal position accumulation (x += dt v; the displacement is x minus a
// stored reference position), the clock, the stable-dt reduction and the
// energy sums stay FP64.
//
// Same algorithm and data flow as the FP64 path (ensc_fp64.cu); operation
// order is free here (FMA contraction on), accuracy is checked against the
// FP64 path by relative displacement error and energy drift.
//
// Element arrays: the bt rows hold A = sum_j B0_j s_j^T (the one-point B0
// rows are A s_j / 8, s_j the node's reference-corner signs) as a float pair,
// 9 hi then 9 lo rows; sigma, qia, eps_p and fe are float; vol0 is double;
// cbrt_v0 is a float copy (in the first ne words of its FP64 storage).
// Node arrays: x double; the u rows hold the reference position x - u
// (double, ENSC_MIXED_UREF); v float with 16-bit residual rows.
#include "ensc_device.cuh"
#include "ensc_kernels.h"
#include "ensc_stage.cuh"

#include <cfloat>

namespace ensc {
namespace {

__device__ __forceinline__ float det3f(const float m[3][3]) {
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

__device__ __forceinline__ float cof3f(const float m[3][3], int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m[i1][j1] * m[i2][j2] - m[i1][j2] * m[i2][j1];
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of NV values into out_slots[i * stride + slot]; values whose bit
// is set in ACC are added to the slot (it accumulates over cycles, one writer
// per slot and pass), the others stored.
template <int NT, int NV, unsigned ACC = 0u>
__device__ __forceinline__ void block_sum_d(double (&v)[NV], double* out_slots, int stride, int slot) {
    __shared__ double red[NV][NT / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double s = warp_sum_d(v[i]);
        if (lane == 0) red[i][wid] = s;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = lane < NT / 32 ? red[i][lane] : 0.0;
            s = warp_sum_d(s);
            if (lane == 0) {
                double* o = out_slots + i * stride + slot;
                if ((ACC >> i) & 1u) atomicAdd(o, s);
                else *o = s;
            }
        }
    }
    __syncthreads();
}

template <int NT>
__device__ __forceinline__ void block_min2_d(double a, double b, unsigned long long* ga, unsigned long long* gb) {
    __shared__ unsigned long long ra[NT / 32], rb[NT / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long x = ord_bits(a), y = ord_bits(b);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long wx = __shfl_xor_sync(0xffffffffu, x, o);
        const unsigned long long wy = __shfl_xor_sync(0xffffffffu, y, o);
        x = wx < x ? wx : x;
        y = wy < y ? wy : y;
    }
    if (lane == 0) {
        ra[wid] = x;
        rb[wid] = y;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < NT / 32; ++i) {
            x = ra[i] < x ? ra[i] : x;
            y = rb[i] < y ? rb[i] : y;
        }
        atomicMin(ga, x);
        atomicMin(gb, y);
    }
    __syncthreads();
}

// Element pass (add_inForce_to_rhs element loop body, exDyna3D.cpp:556-573)
// in FP32.  Node coordinates enter as FP64 offsets from the element's node
// 0; the geometry that every element of a uniform mesh shares (F, edges,
// B0) is carried in FP64 or as float pairs.  Node data are visited twice
// (kinematics, then forces), one component at a time, through the corner
// transforms below.  The hourglass force uses the reassociated sum
// sum_k ATAU(k,j) (QIA(i,k) + CR HIA(i,k))  (exDyna3D.cpp:1053-1070).

// Where one element's inputs are read from: rows of `stride` entries with the
// element at `i` -- the instance's own arrays in global memory, or a
// shared-memory stage that holds a tile of them.
struct MixedSrc {
    const uint32_t* conn;   // [8] rows
    const float* a;         // [18] rows: A hi (3c+m), then A lo
    const double* vol0;
    const float* cb;
    const float* sig;       // [6] rows
    const float* qia;       // [12] rows
    const float* eps;
    int64_t stride, i;
};

__device__ __forceinline__ MixedSrc mixed_src_global(const ElemArrays& E, int64_t e) {
    return MixedSrc{E.conn,
                    static_cast<const float*>(E.bt),
                    E.vol0,
                    reinterpret_cast<const float*>(E.cbrt_v0),
                    static_cast<const float*>(E.sigma),
                    static_cast<const float*>(E.qia),
                    static_cast<const float*>(E.eps_p),
                    E.ne_pad,
                    e};
}

// The one-point B0 row of local node j is A s_j / 8 with A = sum_j B0_j s_j^T
// and s_j the node's reference-corner signs (xi, eta, zeta), Element_HexN8.cpp
// :49-91.

// Sums over the 8 nodes with the signs of the reference corners.  Node j sits
// at corner bits x + 2y + 4z (x set where xi = +1, y for eta, z for zeta);
// for a subset S of {xi, eta, zeta} (bits 0, 1, 2) the coefficient
// c[S] = sum_j (prod_{d in S} sigma_d(j)) a_j, sigma_d(j) = +-1.  The corner
// signs are c[1], c[2], c[4]; the hourglass vectors are
// Gamma = (c[3], -c[6], -c[5], c[7]) (xi eta, -eta zeta, -zeta xi,
// xi eta zeta).  One butterfly of 24 additions gives all of them.
template <typename T>
__device__ __forceinline__ void corner_coeffs(const T (&a)[8], T (&c)[8]) {
    constexpr int kBits[8] = {0, 1, 3, 2, 4, 5, 7, 6};
#pragma unroll
    for (int j = 0; j < 8; ++j) c[kBits[j]] = a[j];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if (!(i & (1 << d))) {
                const T lo = c[i], hi = c[i | (1 << d)];
                c[i] = hi + lo;
                c[i | (1 << d)] = hi - lo;
            }
}

// The other direction: node values a_j = sum_S c[S] prod_{d in S} sigma_d(j)
// (c is overwritten).
template <typename T>
__device__ __forceinline__ void corner_values(T (&c)[8], T (&a)[8]) {
    constexpr int kBits[8] = {0, 1, 3, 2, 4, 5, 7, 6};
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if (!(i & (1 << d))) {
                const T c0 = c[i], c1 = c[i | (1 << d)];
                c[i | (1 << d)] = c0 + c1;
                c[i] = c0 - c1;
            }
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = c[kBits[j]];
}

// One element of the mixed element pass (see the kernel comment below);
// shared by the single-instance, staged and batched kernels.  Inputs come
// from S, outputs go to the instance's arrays at element e.
// PF: node rows prefetched into L1 at the start (bit 0 velocities, bit 1
// coordinate components 1 and 2).
// FOUT: the 24 nodal forces go to fout[3 * 8] (component-major) instead of
// the instance's force array, for the patch assembly.
template <bool PLASTIC, bool INIT, bool SMEM = false, int PF = 0, bool FOUT = false>
__device__ __forceinline__ void element_body_mixed(const ElemArrays& E, const NodeArrays& N, const Material& M,
                                                   const MixedSrc& S, const float dt1, const double dt1d,
                                                   const int64_t e, double& dts, double& len, double& e_int,
                                                   double& e_hg, double& e_vis, int32_t& bad,
                                                   float* fout = nullptr) {
    const int64_t ep = E.ne_pad, np = N.nn_pad, ss = S.stride, si = S.i;
    float* sig = static_cast<float*>(E.sigma);
    float* qia = static_cast<float*>(E.qia);
    float* epsp = static_cast<float*>(E.eps_p);
    float* __restrict__ fe = static_cast<float*>(E.fe);
    const double* __restrict__ X = N.x;
    const float* __restrict__ V = static_cast<const float*>(N.v);
    const float G = M.mc.G;
    const float lam_hi = M.mc.lam_hi, lam_lo = M.mc.lam_lo;
    const float g2_hi = M.mc.g2_hi, g2_lo = M.mc.g2_lo;
    const float rho = M.mc.rho, wos = M.mc.wos;
    const float cvisl = M.mc.cvisl, cvisq = M.mc.cvisq;
    const float y0 = M.mc.y0, H = M.mc.H;
    const float DRc = M.mc.DRc, CRc = M.mc.CRc;
    // A = sum_j B0_j s_j^T as a float pair (hi + lo); B0 enters every
    // product through A, so no FP32 rounding of the reference geometry is
    // shared by all elements of a uniform mesh
    float Ah[3][3], Al[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            Ah[c][m] = ldin<SMEM>(S.a + (3 * c + m) * ss + si);
            Al[c][m] = ldin<SMEM>(S.a + (9 + 3 * c + m) * ss + si);
        }
    uint32_t nk[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) nk[k] = ldin<SMEM>(S.conn + k * ss + si);
    // start the node rows the body reads later on their way into L1
    if (PF & 1) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) prefetch_l1(V + r * np + nk[k]);
    }
    if (PF & 2) {
#pragma unroll
        for (int r = 1; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) prefetch_l1(X + r * np + nk[k]);
    }
    // coordinates relative to node 0, as FP64 differences, one component at a
    // time: hourglass projections TAU x = TAU (x - x0) (the Gamma rows sum to
    // zero) rounded to FP32; the minimum edge and F = sum_j (x_j - x_0) B0_j
    // = (sum_j (x_j - x_0) s_j^T) A^T / 8 (= I + u_e B0^T, as
    // sum_j X0_j B0_j = I and sum_j B0_j = 0) kept in FP64, since on a
    // uniform mesh the FP32 rounding of the spacing would be the same for
    // every element and shift the stiffness and the stable dt of all of them
    float TX[4][3];
    float F[3][3];
    {
        constexpr int A0[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
        constexpr int A1[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
        double e2[12];
        double Gx[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const double* Xr = X + r * np;
            const double xo = Xr[nk[0]];
            double xd[8];
            xd[0] = 0.0;
#pragma unroll
            for (int k = 1; k < 8; ++k) xd[k] = Xr[nk[k]] - xo;
#pragma unroll
            for (int q = 0; q < 12; ++q) {
                const double d = xd[A1[q]] - xd[A0[q]];
                e2[q] = r == 0 ? d * d : fma(d, d, e2[q]);
            }
            double c[8];
            corner_coeffs(xd, c);
            Gx[r][0] = c[1];
            Gx[r][1] = c[2];
            Gx[r][2] = c[4];
            TX[0][r] = static_cast<float>(c[3]);
            TX[1][r] = static_cast<float>(-c[6]);
            TX[2][r] = static_cast<float>(-c[5]);
            TX[3][r] = static_cast<float>(c[7]);
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double t = 0.0;
#pragma unroll
                for (int m = 0; m < 3; ++m)
                    t = fma(Gx[r][m], static_cast<double>(Ah[c][m]) + static_cast<double>(Al[c][m]), t);
                F[r][c] = static_cast<float>(0.125 * t);
            }
        double m = DBL_MAX;
#pragma unroll
        for (int q = 0; q < 12; ++q) m = fmin(m, e2[q]);
        len = sqrt(m);
    }
    const float J = det3f(F);
    if (!(J > 0.f)) bad |= ST_INVERTED;
    const float invdet = 1.f / J;
    float Fi[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Fi[i][j] = cof3f(F, j, i) * invdet;
    // L0 = v_e B0^T = (sum_j v_j s_j^T) A^T / 8, VT = v_e Gamma^T (both from
    // the corner coefficients of each velocity component),
    // NX2 = sum_j |B0_j|^2 = |A|^2 / 8 (sum_j s_j s_j^T = 8 I)
    float L0[3][3], VT[3][4], nx2 = 0.f;
    {
        float Gv[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            float a[8], c[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) a[j] = V[r * np + nk[j]];
            corner_coeffs(a, c);
            Gv[r][0] = c[1];
            Gv[r][1] = c[2];
            Gv[r][2] = c[4];
            VT[r][0] = c[3];
            VT[r][1] = -c[6];
            VT[r][2] = -c[5];
            VT[r][3] = c[7];
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float t = Gv[r][0] * Al[c][0];
                t = fmaf(Gv[r][1], Al[c][1], t);
                t = fmaf(Gv[r][2], Al[c][2], t);
                t = fmaf(Gv[r][0], Ah[c][0], t);
                t = fmaf(Gv[r][1], Ah[c][1], t);
                t = fmaf(Gv[r][2], Ah[c][2], t);
                L0[r][c] = 0.125f * t;
            }
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int m = 0; m < 3; ++m) nx2 = fmaf(Ah[c][m], Ah[c][m], nx2);
        nx2 *= 0.125f;
    }
    // L = L0 F^-1, HIA = VT - L0 TX^T
    float L[3][3], HIA[3][4];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c) L[r][c] = fmaf(L0[r][2], Fi[2][c], fmaf(L0[r][1], Fi[1][c], L0[r][0] * Fi[0][c]));
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            HIA[r][kk] = VT[r][kk] - fmaf(L0[r][2], TX[kk][2], fmaf(L0[r][1], TX[kk][1], L0[r][0] * TX[kk][0]));
    }
    const float vr = L[0][0] + L[1][1] + L[2][2];
    // Jaumann stress update
    float so[6], s[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) so[i] = S.sig[i * ss + si];
    // dt enters the increments as a float pair too: it changes little from
    // cycle to cycle, so its FP32 rounding would repeat with the same sign
    const float dt1_lo = static_cast<float>(dt1d - static_cast<double>(dt1));
    auto incr = [&](float g) { return fmaf(g, dt1, g * dt1_lo); };
    float eps[6] = {incr(L[0][0]), incr(L[1][1]), incr(L[2][2]), incr(0.5f * (L[0][1] + L[1][0])),
                    incr(0.5f * (L[0][2] + L[2][0])), incr(0.5f * (L[1][2] + L[2][1]))};
    {
        const float w0 = incr(0.5f * (L[0][1] - L[1][0]));
        const float w1 = incr(0.5f * (L[0][2] - L[2][0]));
        const float w2 = incr(0.5f * (L[1][2] - L[2][1]));
        const float tr = eps[0] + eps[1] + eps[2];
        // lambda and 2G enter as unevaluated pairs hi + lo of floats: a
        // stiffness rounded to FP32 is off by up to 6e-8 for every element
        // and cycle alike, which shifts all wave speeds and accumulates as
        // phase error; the pair carries the FP64 constants to ~1e-15
        const float lt = fmaf(lam_hi, tr, lam_lo * tr);
        float ge[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) ge[i] = fmaf(g2_hi, eps[i], g2_lo * eps[i]);
        s[0] = so[0] + lt + ge[0] + 2.f * so[3] * w0 + 2.f * so[4] * w1;
        s[1] = so[1] + lt + ge[1] - 2.f * so[3] * w0 + 2.f * so[5] * w2;
        s[2] = so[2] + lt + ge[2] - 2.f * so[4] * w1 - 2.f * so[5] * w2;
        s[3] = so[3] + ge[3] + (so[1] - so[0]) * w0 + so[5] * w1;
        s[4] = so[4] + ge[4] + (so[2] - so[0]) * w1 + so[5] * w0;
        s[5] = so[5] + ge[5] + (so[2] - so[1]) * w2 + so[3] * w1 - so[4] * w0;
    }
    if (PLASTIC) {
        const float pm = (s[0] + s[1] + s[2]) * (1.f / 3.f);
        const float d0 = s[0] - pm, d1 = s[1] - pm, d2 = s[2] - pm;
        const float j2 = 0.5f * (d0 * d0 + d1 * d1 + d2 * d2) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
        const float seq = sqrtf(3.f * j2);
        const float ep_old = S.eps[si];
        const float sy = y0 + H * ep_old;
        if (seq > sy) {
            const float dl = (seq - sy) * M.mc.inv_3gh;
            const float r = 1.f - 3.f * G * dl / seq;
            s[0] = d0 * r + pm;
            s[1] = d1 * r + pm;
            s[2] = d2 * r + pm;
            s[3] *= r;
            s[4] *= r;
            s[5] *= r;
            if (!INIT) epsp[e] = ep_old + dl;
        }
    }
    if (!INIT) {
#pragma unroll
        for (int i = 0; i < 6; ++i) sig[i * ep + e] = s[i];
    }
    const float Vc = static_cast<float>(static_cast<double>(J) * S.vol0[si]);
    {
        float w = 0.f;
#pragma unroll
        for (int i = 0; i < 6; ++i) w += (i < 3 ? 0.5f : 1.0f) * (so[i] + s[i]) * eps[i];
        e_int += static_cast<double>(w * Vc);
    }
    const float DR = DRc * nx2 * Vc * dt1;
    const float cbe = S.cb[si];
    const float CR = CRc * invdet * (cbe * cbe);  // V0 / Vc = 1 / J
    float Gq[3][4];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            const float q = fmaf(DR, HIA[i][kk], S.qia[(4 * i + kk) * ss + si]);
            if (!INIT) qia[(4 * i + kk) * ep + e] = q;
            Gq[i][kk] = fmaf(CR, HIA[i][kk], q);
        }
    const bool visc = !(fabsf(vr) < 1.0e-10f);
    float pv = 0.f;
    if (visc) {
        const float m0 = fminf(vr, 0.f);
        pv = rho * invdet * cbe * (cvisq * cvisq * cbe * vr * m0 - cvisl * wos * vr);
        e_vis += -static_cast<double>(pv * Vc * vr) * dt1d;
    }
    // Z = Vc F^-1 (sigma - p I) - W^T, W = Gq TX
    const float Sp[3][3] = {{s[0] - pv, s[3], s[4]}, {s[3], s[1] - pv, s[5]}, {s[4], s[5], s[2] - pv}};
    float W[3][3], Z[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            W[i][c] = fmaf(Gq[i][3], TX[3][c], fmaf(Gq[i][2], TX[2][c], fmaf(Gq[i][1], TX[1][c], Gq[i][0] * TX[0][c])));
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i)
            Z[c][i] = Vc * fmaf(Fi[c][2], Sp[2][i], fmaf(Fi[c][1], Sp[1][i], Fi[c][0] * Sp[0][i])) - W[i][c];
    {
        // hourglass power sum_j h_j . v_j = Gq : HIA
        float hp = 0.f;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) hp = fmaf(Gq[i][kk], HIA[i][kk], hp);
        e_hg += static_cast<double>(hp) * dt1d;
    }
    // nodal forces f_j = -(B0_j Z) - Gamma_j Gq^T with B0_j Z = s_j^T Y / 8,
    // Y = A^T Z
    // (from a shared-memory stage, A and the connectivity are read again
    // here rather than kept in registers across the stress update)
    constexpr bool kReread = SMEM && ENSC_MIXED_REREAD;
    if (kReread) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                Ah[c][m] = S.a[(3 * c + m) * ss + si];
                Al[c][m] = S.a[(9 + 3 * c + m) * ss + si];
            }
    }
    float Y[3][3];
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float t = Al[0][m] * Z[0][i];
            t = fmaf(Al[1][m], Z[1][i], t);
            t = fmaf(Al[2][m], Z[2][i], t);
            t = fmaf(Ah[0][m], Z[0][i], t);
            t = fmaf(Ah[1][m], Z[1][i], t);
            t = fmaf(Ah[2][m], Z[2][i], t);
            Y[m][i] = 0.125f * t;
        }
    if (kReread) {
#pragma unroll
        for (int k = 0; k < 8; ++k) nk[k] = S.conn[k * ss + si];
    }
    // per force component: the node values of -(B0_j Z) - Gamma_j Gq^T from
    // their corner coefficients (-Y on xi, eta, zeta; -Gq on the hourglass
    // vectors, signed as Gamma)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float c[8] = {0.f,          -Y[0][i],     -Y[1][i],     -Gq[i][0],
                      -Y[2][i],     Gq[i][2],     Gq[i][1],     -Gq[i][3]};
        float f[8];
        corner_values(c, f);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (FOUT) fout[8 * i + j] = f[j];
            else if (E.slot_major) fe[(3 * j + i) * np + nk[j]] = f[j];
            else fe[(3 * j + i) * ep + e] = f[j];
        }
    }
    // element dt (compute_dtStable, exDyna3D.cpp:828-834), with the
    // divisions by wos as products with its reciprocal
    {
        const double m0 = fmin(static_cast<double>(vr), 0.0);
        const double xi = M.cvisl - M.mc.cq2_wos * len * m0;
        dts = (sqrt(1.0 + xi * xi) - xi) * len * M.mc.inv_wos;
    }
    if (!isfinite(dts)) bad |= ST_NONFINITE;
}

template <bool PLASTIC, bool INIT>
__global__ void __launch_bounds__(kElemThreads, ENSC_ELEM_MINB_MIXED)
    k_element_mixed(ElemArrays E, NodeArrays N, Material M, Ctl* ctl, Partials P) {
    if (ctl->done) return;
    const float dt1 = INIT ? 0.f : static_cast<float>(ctl->dt_i_1);
    const double dt1d = INIT ? 0.0 : ctl->dt_i_1;
    const int64_t ne = E.ne;
    double e_int = 0.0, e_hg = 0.0, e_vis = 0.0;
    double dts_min = DBL_MAX, len_min = DBL_MAX;
    int32_t bad = 0;

    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < ne; e += stride) {
        double dts, len;
        element_body_mixed<PLASTIC, INIT>(E, N, M, mixed_src_global(E, e), dt1, dt1d, e, dts, len, e_int, e_hg, e_vis,
                                          bad);
        dts_min = fmin(dts_min, dts);
        len_min = fmin(len_min, len);
    }
    if (bad) atomicOr(&ctl->status, bad);
    block_min2_d<kElemThreads>(dts_min, len_min, &ctl->dts_next, &ctl->len_min);
    if (!INIT) {
        double v3[3] = {e_int, e_hg, e_vis};
        block_sum_d<kElemThreads, 3, 7u>(v3, P.elem, P.n_elem_blocks, blockIdx.x);
    }
}

// ---- staged element pass ------------------------------------------------
// Each block walks tiles of kStageTile consecutive elements.  Thread 0 copies
// a tile's streamed inputs -- connectivity, the B0 matrix A (hi and lo),
// sigma, QIA, cbrt(V0), eps_p and V0 -- into one of two
// shared-memory stages with bulk copies, one tile ahead of the compute; the
// block then evaluates the tile with element_body_mixed reading those inputs
// from the stage while the next tile's copies are in flight.  Node data are
// gathered from global memory as in the unstaged pass, and all outputs are
// written there.
constexpr int kStageTile = ENSC_STAGE_TILE_MIXED;
// stage: 46 rows of 4-byte words (8 conn, 18 A, 6 sigma, 12 QIA, cbrt(V0),
// eps_p), then V0 as a row of doubles
constexpr int kStageWordRows = 46;
constexpr uint32_t kStageV0Off = kStageWordRows * kStageTile * 4;
constexpr uint32_t kStageBytes = kStageV0Off + kStageTile * 8;
constexpr size_t kStageSmem = 2 * static_cast<size_t>(kStageBytes) + 16;  // two stages, two barriers

// word row r of the stage in global memory
__device__ __forceinline__ const float* stage_row(const ElemArrays& E, int r) {
    const int64_t ep = E.ne_pad;
    if (r < 8) return reinterpret_cast<const float*>(E.conn + r * ep);
    if (r < 26) return static_cast<const float*>(E.bt) + (r - 8) * ep;
    if (r < 32) return static_cast<const float*>(E.sigma) + (r - 26) * ep;
    if (r < 44) return static_cast<const float*>(E.qia) + (r - 32) * ep;
    if (r == 44) return reinterpret_cast<const float*>(E.cbrt_v0);
    return static_cast<const float*>(E.eps_p);
}

// Warp 0 copies the tile starting at element `base` into the stage at
// shared address dst, completing on bar: lane 0 arms the barrier with the
// byte count, then the lanes start the row copies between them.  The rows
// are padded to a multiple of 32 entries and start 256-byte aligned, so
// every copy is 16-byte aligned and a multiple of 128 bytes long.
template <bool PLASTIC>
__device__ __forceinline__ uint32_t stage_count(const ElemArrays& E, int64_t base) {
    const int64_t left = E.ne_pad - base;
    return static_cast<uint32_t>(left < kStageTile ? left : kStageTile);
}
template <bool PLASTIC>
__device__ __forceinline__ uint32_t stage_tx_bytes(uint32_t cnt) {
    constexpr int rows = PLASTIC ? kStageWordRows : kStageWordRows - 1;  // eps_p last, J2 only
    return rows * cnt * 4u + cnt * 8u;
}
template <bool PLASTIC>
__device__ __forceinline__ void stage_issue(const ElemArrays& E, uint32_t dst, uint32_t bar, int64_t base, int lane) {
    constexpr int rows = PLASTIC ? kStageWordRows : kStageWordRows - 1;
    const uint32_t cnt = stage_count<PLASTIC>(E, base);
    if (lane == 0) mbar_arrive_expect_tx(bar, stage_tx_bytes<PLASTIC>(cnt));
    __syncwarp();
    fence_proxy_async_smem();  // the block's reads of this stage come before the copies into it
    for (int r = lane; r <= rows; r += 32) {
        if (r < rows) bulk_g2s(dst + r * (kStageTile * 4u), stage_row(E, r) + base, cnt * 4u, bar);
        else bulk_g2s(dst + kStageV0Off, E.vol0 + base, cnt * 8u, bar);
    }
}

template <bool PLASTIC>
__global__ void __launch_bounds__(kStageTile, ENSC_STAGE_MINB_MIXED)
    k_element_mixed_staged(ElemArrays E, NodeArrays N, Material M, Ctl* ctl, Partials P) {
    if (ctl->done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    const float dt1 = static_cast<float>(ctl->dt_i_1);
    const double dt1d = ctl->dt_i_1;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t stage0 = smem_addr(smem);
    const uint32_t bar0 = stage0 + 2 * kStageBytes;
    const int64_t ntiles = (E.ne + kStageTile - 1) / kStageTile;
    const int64_t gstride = gridDim.x;
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (wid == 0) {
        for (int s = 0; s < 2; ++s) {
            const int64_t t = blockIdx.x + s * gstride;
            if (t < ntiles) stage_issue<PLASTIC>(E, stage0 + s * kStageBytes, bar0 + 8 * s, t * kStageTile, lane);
        }
    }
    double e_int = 0.0, e_hg = 0.0, e_vis = 0.0;
    double dts_min = DBL_MAX, len_min = DBL_MAX;
    int32_t bad = 0;
    bool timed_out = false;
    int it = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gstride, ++it) {
        const int s = it & 1;
        const uint32_t bar = bar0 + 8 * s;
        const bool ok = mbar_wait_bounded(bar, (it >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
        const int64_t e = t * kStageTile + tid;
        if (e < E.ne) {
            const float* st = reinterpret_cast<const float*>(smem + s * kStageBytes);
            const MixedSrc S{reinterpret_cast<const uint32_t*>(st),
                             st + 8 * kStageTile,
                             reinterpret_cast<const double*>(smem + s * kStageBytes + kStageV0Off),
                             st + 44 * kStageTile,
                             st + 26 * kStageTile,
                             st + 32 * kStageTile,
                             st + 45 * kStageTile,
                             kStageTile,
                             tid};
            double dts, len;
            element_body_mixed<PLASTIC, false, true, ENSC_MIXED_PREFETCH>(E, N, M, S, dt1, dt1d, e, dts, len, e_int,
                                                                          e_hg, e_vis, bad);
            dts_min = fmin(dts_min, dts);
            len_min = fmin(len_min, len);
        }
        __syncthreads();  // the block is done with stage s
        const int64_t tn = t + 2 * gstride;
        if (wid == 0 && tn < ntiles) stage_issue<PLASTIC>(E, stage0 + s * kStageBytes, bar, tn * kStageTile, lane);
    }
    if (timed_out) {
        // record the failure and let the copies this block started land
        // (bounded) before its shared memory is released
        if (tid == 0) {
            atomicOr(&ctl->status, ST_TIMEOUT);
            for (int k = 0; k < 2; ++k) {
                const int itk = it + k;
                if (blockIdx.x + itk * gstride < ntiles) mbar_wait_bounded(bar0 + 8 * (itk & 1), (itk >> 1) & 1);
            }
        }
        __syncthreads();
    }
    if (bad) atomicOr(&ctl->status, bad);
    block_min2_d<kStageTile>(dts_min, len_min, &ctl->dts_next, &ctl->len_min);
    double v3[3] = {e_int, e_hg, e_vis};
    block_sum_d<kStageTile, 3, 7u>(v3, P.elem, P.n_elem_blocks, blockIdx.x);
}

// ---- staged element pass with patch assembly ----------------------------
// k_element_mixed_staged with one patch per tile.  After its element body a
// thread holds its element's 24 nodal forces; once the whole block is done
// with the stage's inputs, the forces go into the stage's memory as
// [3][8 slots][kStageTile elements], and the block sums each of the patch's
// nodes over its incidences in slot order (starting from zero) and writes the
// node's partial to PA.pf.  INIT: the init force pass (dt = 0, no state
// written, no energy).
static_assert(kStageTile == kPatchElems, "one patch per staged tile");
static_assert(3u * 8u * kStageTile * 4u <= kStageBytes, "the element forces fit in a stage");

__device__ __forceinline__ void patch_partials(const PatchArrays& E, const float* sf, int64_t t, int tid) {
    const uint32_t q0 = __ldg(E.pf_off + t), q1 = __ldg(E.pf_off + t + 1);
    for (uint32_t q = q0 + tid; q < q1; q += kStageTile) {
        const uint32_t a = __ldg(E.pinc_off + q), b = __ldg(E.pinc_off + q + 1);
        float f0 = 0.f, f1 = 0.f, f2 = 0.f;
        for (uint32_t r = a; r < b; ++r) {
            const uint32_t u = __ldg(E.pinc + r);
            const uint32_t col = (u & 7u) * kStageTile + (u >> 3);
            f0 += sf[col];
            f1 += sf[8 * kStageTile + col];
            f2 += sf[16 * kStageTile + col];
        }
        E.pf[q] = f0;
        E.pf[E.pf_pad + q] = f1;
        E.pf[2 * E.pf_pad + q] = f2;
    }
}

template <bool PLASTIC, bool INIT>
__global__ void __launch_bounds__(kStageTile, ENSC_STAGE_MINB_MIXED)
    k_element_mixed_patch(ElemArrays E, NodeArrays N, Material M, Ctl* ctl, Partials P, PatchArrays PA) {
    if (ctl->done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    const float dt1 = INIT ? 0.f : static_cast<float>(ctl->dt_i_1);
    const double dt1d = INIT ? 0.0 : ctl->dt_i_1;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t stage0 = smem_addr(smem);
    const uint32_t bar0 = stage0 + 2 * kStageBytes;
    const int64_t ntiles = (E.ne + kStageTile - 1) / kStageTile;
    const int64_t gstride = gridDim.x;
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (wid == 0) {
        for (int s = 0; s < 2; ++s) {
            const int64_t t = blockIdx.x + s * gstride;
            if (t < ntiles) stage_issue<PLASTIC>(E, stage0 + s * kStageBytes, bar0 + 8 * s, t * kStageTile, lane);
        }
    }
    double e_int = 0.0, e_hg = 0.0, e_vis = 0.0;
    double dts_min = DBL_MAX, len_min = DBL_MAX;
    int32_t bad = 0;
    bool timed_out = false;
    int it = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gstride, ++it) {
        const int s = it & 1;
        const uint32_t bar = bar0 + 8 * s;
        const bool ok = mbar_wait_bounded(bar, (it >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
        const int64_t e = t * kStageTile + tid;
        const bool live = e < E.ne;
        float fo[24];
        if (live) {
            const float* st = reinterpret_cast<const float*>(smem + s * kStageBytes);
            const MixedSrc S{reinterpret_cast<const uint32_t*>(st),
                             st + 8 * kStageTile,
                             reinterpret_cast<const double*>(smem + s * kStageBytes + kStageV0Off),
                             st + 44 * kStageTile,
                             st + 26 * kStageTile,
                             st + 32 * kStageTile,
                             st + 45 * kStageTile,
                             kStageTile,
                             tid};
            double dts, len;
            element_body_mixed<PLASTIC, INIT, true, ENSC_MIXED_PREFETCH, true>(E, N, M, S, dt1, dt1d, e, dts, len,
                                                                               e_int, e_hg, e_vis, bad, fo);
            dts_min = fmin(dts_min, dts);
            len_min = fmin(len_min, len);
        }
        __syncthreads();  // the stage's inputs are consumed
        float* sf = reinterpret_cast<float*>(smem + s * kStageBytes);
        if (live) {
#pragma unroll
            for (int i = 0; i < 24; ++i) sf[i * kStageTile + tid] = fo[i];
        }
        __syncthreads();
        patch_partials(PA, sf, t, tid);
        __syncthreads();  // the block is done with stage s
        const int64_t tn = t + 2 * gstride;
        if (wid == 0 && tn < ntiles) stage_issue<PLASTIC>(E, stage0 + s * kStageBytes, bar, tn * kStageTile, lane);
    }
    if (timed_out) {
        if (tid == 0) {
            atomicOr(&ctl->status, ST_TIMEOUT);
            for (int k = 0; k < 2; ++k) {
                const int itk = it + k;
                if (blockIdx.x + itk * gstride < ntiles) mbar_wait_bounded(bar0 + 8 * (itk & 1), (itk >> 1) & 1);
            }
        }
        __syncthreads();
    }
    if (bad) atomicOr(&ctl->status, bad);
    block_min2_d<kStageTile>(dts_min, len_min, &ctl->dts_next, &ctl->len_min);
    if (!INIT) {
        double v3[3] = {e_int, e_hg, e_vis};
        block_sum_d<kStageTile, 3, 7u>(v3, P.elem, P.n_elem_blocks, blockIdx.x);
    }
}

// One node's force under the patch assembly: its partials in patch order,
// from zero.
__device__ __forceinline__ void patch_gather(const PatchArrays& PA, int64_t n, float (&f)[3]) {
    const int64_t pp = PA.pf_pad;
    for (uint32_t r = __ldg(PA.nptr + n), b = __ldg(PA.nptr + n + 1); r < b; ++r) {
        const uint32_t q = __ldg(PA.nent + r);
        f[0] += __ldg(PA.pf + q);
        f[1] += __ldg(PA.pf + pp + q);
        f[2] += __ldg(PA.pf + 2 * pp + q);
    }
}

#if !ENSC_MIXED_VLO
// v + (dt_i + dt_i_1) / 2 * f * M^-1 in FP32 with the half step and the
// inverse mass as float pairs: both are the same for many nodes and cycles,
// so their FP32 rounding would scale all accelerations alike.
__device__ __forceinline__ float velocity_update(float vo, float f, double im, float hdt, float hdt_lo) {
    const float im_hi = static_cast<float>(im);
    const float im_lo = static_cast<float>(im - static_cast<double>(im_hi));
    const float acc = fmaf(f, im_hi, f * im_lo);
    return fmaf(hdt, acc, fmaf(hdt_lo, acc, vo));
}
#endif

// The velocity update in FP64 on the split velocity (hi float + 16-bit
// residual, v_join / v_split): v + (dt_i + dt_i_1) / 2 * a with the FP32
// acceleration a = f M^-1 (inverse mass as a float pair); returns the new
// velocity as a double and its split form.
__device__ __forceinline__ double velocity_update_split(double vo, float f, double im, double hdt, float& hi,
                                                        int16_t& lo) {
    const float im_hi = static_cast<float>(im);
    const float im_lo = static_cast<float>(im - static_cast<double>(im_hi));
    const float acc = fmaf(f, im_hi, f * im_lo);
    const double vn = fma(hdt, static_cast<double>(acc), vo);
    v_split(vn, hi, lo);
    return vn;
}

// One node of the mixed node pass; shared by the single-instance and
// batched kernels.
__device__ __forceinline__ void node_body_mixed(const ElemArrays& E, const NodeArrays& N, const Material& M,
                                                const double dt_i, const double dt_i_1, const double amp, const int64_t n,
                                                double& kin, double& wext, int32_t& bad) {
    const int64_t np = N.nn_pad, ep = E.ne_pad;
    const float* __restrict__ fe = static_cast<const float*>(E.fe);
    float* __restrict__ V = static_cast<float*>(N.v);
    [[maybe_unused]] const float hdt = static_cast<float>(0.5 * (dt_i + dt_i_1));
    [[maybe_unused]] const float hdt_lo = static_cast<float>(0.5 * (dt_i + dt_i_1) - static_cast<double>(hdt));
    const double dt_avg = 0.5 * (dt_i + dt_i_1);

    float f[3] = {0.f, 0.f, 0.f};
    if (E.slot_major) {
        const uint32_t msk = N.slot_mask[n];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if ((msk >> k) & 1u) {
#pragma unroll
                for (int c = 0; c < 3; ++c) f[c] += fe[(3 * k + c) * np + n];
            }
        }
    } else if (N.csr_ptr == nullptr) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t el = __ldg(N.ell + k * np + n);
            if (el != ENSC_NONE) {
#pragma unroll
                for (int c = 0; c < 3; ++c) f[c] += fe[(3 * k + c) * ep + el];
            }
        }
    } else {
        for (int64_t i = N.csr_ptr[n]; i < N.csr_ptr[n + 1]; ++i) {
            const uint32_t ent = N.csr_ent[i];
            const int k = static_cast<int>(ent & 7u);
            const uint32_t el = ent >> 3;
#pragma unroll
            for (int c = 0; c < 3; ++c) f[c] += fe[(3 * k + c) * ep + el];
        }
    }
    const double im = N.inv_mass[n];
    const uint32_t code = N.bc[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float a = f[c];
        float g = 0.f;
        if (M.gravity_on) {
            g = static_cast<float>(amp * M.gravity_value * M.gravity_dir[c] / im);
            a += g;
        }
        const uint32_t cc = (code >> (2 * c)) & 3u;
        float r = 0.f, rf = 0.f;
        if (cc & 2u) {
            r = -a;
            a = 0.f;
        }
        if ((cc & 1u) && a != 0.f) {
            rf = -a;
            r = -a;
            a = 0.f;
        }
        if (cc) N.rf[c * np + n] = static_cast<double>(rf);
#if ENSC_MIXED_VLO
        int16_t* VL = v_lo_rows(N.v, np);
        const double vod = v_join(V[c * np + n], VL[c * np + n]);
        float vn;
        int16_t vl;
        const double vnd = velocity_update_split(vod, a, im, dt_avg, vn, vl);
        V[c * np + n] = vn;
        VL[c * np + n] = vl;
#else
        const float vo = V[c * np + n];
        const float vn = velocity_update(vo, a, im, hdt, hdt_lo);
        V[c * np + n] = vn;
        const double vnd = static_cast<double>(vn);
        const double vod = static_cast<double>(vo);
#endif
        if (!ENSC_MIXED_UREF) N.u[c * np + n] += dt_i * vnd;
        N.x[c * np + n] += dt_i * vnd;
        wext += static_cast<double>(g + r) * dt_avg * 0.5 * (vod + vnd);
        kin += 0.5 * (vnd * vnd) / im;
        if (!isfinite(vnd)) bad |= ST_NONFINITE;
    }
}

// W consecutive nodes of the mixed node pass with 16-byte row accesses
// (float4 force slots and velocities, pairs of doubles for x and the
// inverse mass); per node the arithmetic of node_body_mixed.  Slots the mask
// marks empty are skipped, or (ENSC_NODE_ALL_SLOTS) summed as the zeros they
// hold: the slot-major rows start zeroed and only the slot's element writes
// them.  Nodes at or past nn (row padding) are loaded and stored back
// unchanged.
template <int W, bool PATCH>
__device__ __forceinline__ void node_group_mixed(const NodeView& N, const double dt_i, const double dt_i_1,
                                                 const double amp, const int64_t n0, double& kin, double& wext,
                                                 int32_t& bad) {
    const int64_t np = N.np, nn = N.nn;
    const float* __restrict__ fe = static_cast<const float*>(N.fe);
    float* __restrict__ V = static_cast<float*>(N.v);
    [[maybe_unused]] const float hdt = static_cast<float>(0.5 * (dt_i + dt_i_1));
    [[maybe_unused]] const float hdt_lo = static_cast<float>(0.5 * (dt_i + dt_i_1) - static_cast<double>(hdt));
    const double dt_avg = 0.5 * (dt_i + dt_i_1);
#if ENSC_NODE_LOAD_FIRST
    // the nodes' own rows first, so that their loads are in flight with the
    // force slots'
    double im[W];
    ld_row<W>(N.inv_mass + n0, im);
    const uint32_t code = ld_bytes<W>(N.bc + n0);
    float vo3[3][W];
    double xo3[3][W];
    int16_t lo3[3][W];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        ld_row<W>(V + c * np + n0, vo3[c]);
        ld_row<W>(N.x + c * np + n0, xo3[c]);
        ld_row<W>(v_lo_rows(N.v, np) + c * np + n0, lo3[c]);
    }
#endif
    float f[3][W];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int j = 0; j < W; ++j) f[c][j] = 0.f;
    if constexpr (PATCH) {
        // patch assembly: the node's partials in patch order
        uint32_t lo[W], bnd[W + 1];
        ld_row<W>(N.nptr + n0, lo);
#pragma unroll
        for (int j = 0; j < W; ++j) bnd[j] = lo[j];
        bnd[W] = __ldg(N.nptr + n0 + W);
        const int64_t pp = N.pf_pad;
#pragma unroll
        for (int j = 0; j < W; ++j) {
            for (uint32_t r = bnd[j]; r < bnd[j + 1]; ++r) {
                const uint32_t q = __ldg(N.nent + r);
                f[0][j] += __ldg(N.pf + q);
                f[1][j] += __ldg(N.pf + pp + q);
                f[2][j] += __ldg(N.pf + 2 * pp + q);
            }
        }
    } else {
        const uint32_t msk = ENSC_NODE_ALL_SLOTS ? 0xffffffffu : ld_bytes<W>(N.slot_mask + n0);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            uint32_t sel = 0;
#pragma unroll
            for (int j = 0; j < W; ++j) sel |= ((msk >> (8 * j + k)) & 1u) << j;
            if (sel) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    float r[W];
                    ld_row<W>(fe + (3 * k + c) * np + n0, r);
#pragma unroll
                    for (int j = 0; j < W; ++j)
                        if ((sel >> j) & 1u) f[c][j] += r[j];
                }
            }
        }
    }
#if !ENSC_NODE_LOAD_FIRST
    double im[W];
    ld_row<W>(N.inv_mass + n0, im);
    const uint32_t code = ld_bytes<W>(N.bc + n0);
#endif
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float vo[W], vn[W];
        double uo[W], xo[W], un[W], xn[W];
#if ENSC_MIXED_VLO
        int16_t* VL = v_lo_rows(N.v, np);
        int16_t lo[W], ln[W];
#endif
#if ENSC_NODE_LOAD_FIRST
#pragma unroll
        for (int j = 0; j < W; ++j) {
            vo[j] = vo3[c][j];
            xo[j] = xo3[c][j];
            lo[j] = lo3[c][j];
        }
#else
        ld_row<W>(V + c * np + n0, vo);
        ld_row<W>(N.x + c * np + n0, xo);
#if ENSC_MIXED_VLO
        ld_row<W>(VL + c * np + n0, lo);
#endif
#endif
        if (!ENSC_MIXED_UREF) ld_row<W>(N.u + c * np + n0, uo);
#pragma unroll
        for (int j = 0; j < W; ++j) {
            vn[j] = vo[j];
#if ENSC_MIXED_VLO
            ln[j] = lo[j];
#endif
            if (!ENSC_MIXED_UREF) un[j] = uo[j];
            xn[j] = xo[j];
            if (n0 + j >= nn) continue;
            float a = f[c][j];
            float g = 0.f;
            if (N.gravity_on) {
                g = static_cast<float>(amp * N.gravity_value * N.gravity_dir[c] / im[j]);
                a += g;
            }
            const uint32_t cc = (code >> (8 * j + 2 * c)) & 3u;
            float r = 0.f, rf = 0.f;
            if (cc & 2u) {
                r = -a;
                a = 0.f;
            }
            if ((cc & 1u) && a != 0.f) {
                rf = -a;
                r = -a;
                a = 0.f;
            }
            if (cc) N.rf[c * np + n0 + j] = static_cast<double>(rf);
#if ENSC_MIXED_VLO
            const double vod = v_join(vo[j], lo[j]);
            const double vnd = velocity_update_split(vod, a, im[j], dt_avg, vn[j], ln[j]);
#else
            vn[j] = velocity_update(vo[j], a, im[j], hdt, hdt_lo);
            const double vnd = static_cast<double>(vn[j]);
            const double vod = static_cast<double>(vo[j]);
#endif
            if (!ENSC_MIXED_UREF) un[j] = uo[j] + dt_i * vnd;
            xn[j] = xo[j] + dt_i * vnd;
            wext += static_cast<double>(g + r) * dt_avg * 0.5 * (vod + vnd);
            kin += 0.5 * (vnd * vnd) / im[j];
            if (!isfinite(vnd)) bad |= ST_NONFINITE;
        }
        st_row<W>(V + c * np + n0, vn);
#if ENSC_MIXED_VLO
        st_row<W>(VL + c * np + n0, ln);
#endif
        if (!ENSC_MIXED_UREF) st_row<W>(N.u + c * np + n0, un);
        st_row<W>(N.x + c * np + n0, xn);
    }
}

// Node pass in mixed precision: FP32 slot-ordered gather and acceleration,
// FP32 velocity, FP64 position accumulation and energy (the u rows hold the
// reference position x - u and are not touched: ENSC_MIXED_UREF).
// PATCH: the instance uses the patch assembly (one instantiation each, so
// the slot-assembly pass carries no code of the other).
template <bool PATCH>
__global__ void __launch_bounds__(kNodeThreads, ENSC_NODE_MINB_MIXED) k_node_mixed(ElemArrays E, NodeArrays N, Material M, Ctl* ctl,
                                                             Partials P, PatchArrays PA) {
    if (ctl->done) return;
    double dt_i;
    const double dt_i_1 = ctl->dt_i_1;
    if (ctl->dt_final) {
        dt_i = ctl->dt_i;
    } else {
        double d = bits_ord(ctl->len_min) / ctl->wos;
        d = d < ctl->dts_cur ? d : ctl->dts_cur;
        dt_i = d * ctl->factor;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (!(dt_i > 0.0) || !isfinite(dt_i)) atomicOr(&ctl->status, ST_BAD_DT);
        if (!ctl->dt_final) ctl->dt_i = dt_i;
        ctl->cycles_done += 1;
        ctl->energy_pending = 1;
    }
    const int64_t nn = N.nn;
    const double amp = (M.gravity_on && M.amp_n > 0) ? gravity_amplitude(M.amp, M.amp_n, ctl->time, dt_i) : 1.0;
    double kin = 0.0, wext = 0.0;
    int32_t bad = 0;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (E.slot_major && E.tiles_aligned) {
        constexpr int W = kNodeGroupMixed;
        const NodeView nv = node_view(E, N, M, ctl, &PA);
        for (int64_t g = t0; g * W < nn; g += stride)
            node_group_mixed<W, PATCH>(nv, dt_i, dt_i_1, amp, g * W, kin, wext, bad);
    } else {
        for (int64_t n = t0; n < nn; n += stride) node_body_mixed(E, N, M, dt_i, dt_i_1, amp, n, kin, wext, bad);
    }
    if (bad) atomicOr(&ctl->status, bad);
    double v2[2] = {kin, wext};
    block_sum_d<kNodeThreads, 2, 2u>(v2, P.node, P.n_node_blocks, blockIdx.x);
}


// The last cycle's acceleration in mixed precision (see k_acceleration in
// the FP64 stepper): the FP32 force sum, gravity and the FP32 acceleration
// f M^-1 that the mixed node pass feeds into the velocity update, written
// as doubles, interleaved xyz per node.
__global__ void __launch_bounds__(kNodeThreads) k_acceleration_mixed(PatchArrays PA, ElemArrays E, NodeArrays N, Material M,
                                                                     const Ctl* ctl, double* a_out) {
    const int64_t np = N.nn_pad, ep = E.ne_pad;
    const float* __restrict__ fe = static_cast<const float*>(E.fe);
    const bool grouped = E.slot_major && E.tiles_aligned;
    const double amp = (M.gravity_on && M.amp_n > 0) ? gravity_amplitude(M.amp, M.amp_n, ctl->time, ctl->dt_i) : 1.0;
    for (int64_t n = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; n < N.nn;
         n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        float f[3] = {0.f, 0.f, 0.f};
        if (PA.pf) {
            patch_gather(PA, n, f);
        } else if (E.slot_major) {
            const uint32_t msk = grouped ? 0xffu : N.slot_mask[n];
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if ((msk >> k) & 1u) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) f[c] += fe[(3 * k + c) * np + n];
                }
        } else if (N.csr_ptr == nullptr) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t el = N.ell[k * np + n];
                if (el != ENSC_NONE) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) f[c] += fe[(3 * k + c) * ep + el];
                }
            }
        } else {
            for (int64_t i = N.csr_ptr[n]; i < N.csr_ptr[n + 1]; ++i) {
                const uint32_t ent = N.csr_ent[i];
                const int k = static_cast<int>(ent & 7u);
                const uint32_t el = ent >> 3;
#pragma unroll
                for (int c = 0; c < 3; ++c) f[c] += fe[(3 * k + c) * ep + el];
            }
        }
        const double im = N.inv_mass[n];
        const float im_hi = static_cast<float>(im);
        const float im_lo = static_cast<float>(im - static_cast<double>(im_hi));
        const uint32_t code = N.bc[n];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float a = f[c];
            if (M.gravity_on) a += static_cast<float>(amp * M.gravity_value * M.gravity_dir[c] / im);
            const uint32_t cc = (code >> (2 * c)) & 3u;
            if (cc & 2u) a = 0.f;
            if ((cc & 1u) && a != 0.f) a = 0.f;
            a_out[3 * n + c] = static_cast<double>(fmaf(a, im_hi, a * im_lo));
        }
    }
}

// ---- batched instances --------------------------------------------------------
// Element tiles of kStageTile elements and node tiles of 32 * kNodeGroupBatchMixed
// nodes, each inside one instance whose arrays, material and control block
// come from the instance table.  The element pass runs the staged pipeline
// over the tile list, one tile per block at a time; the node pass gives each
// node tile to one warp.  Each tile accumulates its work terms across
// cycles (one owner per tile and pass) and keeps its latest kinetic energy;
// k_fold_batch folds them per instance in tile order, so the totals do not
// depend on scheduling.
__device__ __forceinline__ double warp_sum_b(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// A batch stage: the single-instance stage, then the tile's instance
// descriptor, its element-pass scalars (StageHdr), the TileInfo the filling
// warp writes, and the ETileSrc record of the tile that uses the stage next.
// Every tile is copied whole whether or not its instance runs this cycle;
// the consumer skips the tiles of instances that do not.
constexpr uint32_t kDescBytes = sizeof(InstanceDesc);
constexpr uint32_t kBatchDescOff = kStageBytes;
constexpr uint32_t kBatchHdrOff = kBatchDescOff + kDescBytes;
constexpr uint32_t kBatchInfoOff = kBatchHdrOff + sizeof(StageHdr);
constexpr uint32_t kBatchNextOff = kBatchInfoOff + sizeof(TileInfo);
constexpr uint32_t kBatchStageBytes = (kBatchNextOff + sizeof(ETileSrc) + 127) / 128 * 128;
constexpr size_t kBatchStageSmem = 2 * static_cast<size_t>(kBatchStageBytes) + 16;
static_assert(kDescBytes % 16 == 0 && sizeof(StageHdr) == 16 && sizeof(TileInfo) == 16, "16-byte copies");

// word row r of a batch tile in global memory
__device__ __forceinline__ const void* tile_row(const ETileSrc& src, int r) {
    const int64_t ep = src.ne_pad;
    if (r < 8) return static_cast<const uint32_t*>(src.conn) + r * ep;
    if (r < 26) return static_cast<const float*>(src.bt) + (r - 8) * ep;
    if (r < 32) return static_cast<const float*>(src.sigma) + (r - 26) * ep;
    if (r < 44) return static_cast<const float*>(src.qia) + (r - 32) * ep;
    if (r == 44) return src.cbrt_v0;
    return src.eps_p;
}

// Warp 0 fills a stage with the tile `src` describes (and the record of tile
// t_next, if there is one): lane 0 writes the TileInfo and arms the barrier
// with the byte count, then the lanes start the copies between them.
__device__ __forceinline__ void batch_stage_issue(const BatchTables& T, const ETileSrc& src, int64_t t_next,
                                                  int64_t ntiles, unsigned char* stage, uint32_t dst, uint32_t bar,
                                                  int lane) {
    const uint32_t cnt = static_cast<uint32_t>(src.cnt);
    const bool next = t_next < ntiles;
    if (lane == 0) {
        TileInfo* ti = reinterpret_cast<TileInfo*>(stage + kBatchInfoOff);
        ti->slot = src.slot;
        ti->base = src.base;
        mbar_arrive_expect_tx(bar, kStageWordRows * cnt * 4u + cnt * 8u + kDescBytes + sizeof(StageHdr) +
                                       (next ? sizeof(ETileSrc) : 0u));
    }
    __syncwarp();
    fence_proxy_async_smem();  // the block's reads of this stage come before the copies into it
    for (int r = lane; r < kStageWordRows + 4; r += 32) {
        if (r < kStageWordRows) bulk_g2s(dst + r * (kStageTile * 4u), tile_row(src, r), cnt * 4u, bar);
        else if (r == kStageWordRows) bulk_g2s(dst + kStageV0Off, src.vol0, cnt * 8u, bar);
        else if (r == kStageWordRows + 1) bulk_g2s(dst + kBatchDescOff, T.desc + src.slot, kDescBytes, bar);
        else if (r == kStageWordRows + 2) bulk_g2s(dst + kBatchHdrOff, T.sparam + src.slot, sizeof(StageHdr), bar);
        else if (next) bulk_g2s(dst + kBatchNextOff, T.etile_src + t_next, sizeof(ETileSrc), bar);
    }
}

// EPT elements per thread: the block has kStageTile / EPT threads, and each
// thread evaluates elements tid, tid + kStageTile / EPT, ... of a tile in
// turn (a tuning choice; EPT > 1 only under the slot assembly).  PATCH: the
// batch's instances use the patch assembly (a batch has one assembly).
template <int EPT, bool PATCH>
__global__ void __launch_bounds__(kStageTile / EPT, ENSC_BATCH_MINB_MIXED) k_element_batch_mixed(BatchTables T) {
    static_assert(EPT == 1 || !PATCH, "the patch sums take one element per thread");
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int NW = kStageTile / 32;  // energy partial slots per tile
    constexpr int NT = kStageTile / EPT;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t stage0 = smem_addr(smem);
    const uint32_t bar0 = stage0 + 2 * kBatchStageBytes;
    const int64_t ntiles = T.counts[0];
    const int64_t gstride = gridDim.x;
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (wid == 0) {
        for (int s = 0; s < 2; ++s) {
            const int64_t t = blockIdx.x + s * gstride;
            if (t < ntiles) {
                const ETileSrc src = T.etile_src[t];
                batch_stage_issue(T, src, t + 2 * gstride, ntiles, smem + s * kBatchStageBytes,
                                  stage0 + s * kBatchStageBytes, bar0 + 8 * s, lane);
            }
        }
    }
    // the current run: instance slot, first tile, control block, liveness
    int run_slot = -1;
    int64_t run_tile = 0;
    Ctl* run_ctl = nullptr;
    bool run_live = false;
    double ei = 0.0, eh = 0.0, ev = 0.0, dts = DBL_MAX, len = DBL_MAX;
    int32_t bad = 0;
    auto flush = [&]() {
        ei = warp_sum_b(ei);
        eh = warp_sum_b(eh);
        ev = warp_sum_b(ev);
        const unsigned long long dmin = warp_min_u64(ord_bits(dts));
        const unsigned long long lmin = warp_min_u64(ord_bits(len));
        bad = static_cast<int32_t>(__reduce_or_sync(0xffffffffu, static_cast<unsigned>(bad)));
        if (run_live && lane == 0) {
            double* part = T.etile_part + 3 * (run_tile * NW + wid);
            // one writer per slot and pass: the reductions (no return value)
            // add in cycle order without a round trip
            atomicAdd(part + 0, ei);
            atomicAdd(part + 1, eh);
            atomicAdd(part + 2, ev);
            atomicMin(&run_ctl->dts_next, dmin);
            atomicMin(&run_ctl->len_min, lmin);
            if (bad) atomicOr(&run_ctl->status, bad);
        }
        ei = eh = ev = 0.0;
        dts = len = DBL_MAX;
        bad = 0;
    };
    bool timed_out = false;
    int it = 0;
    int64_t t = blockIdx.x;
    for (; t < ntiles; t += gstride, ++it) {
        const int s = it & 1;
        const uint32_t bar = bar0 + 8 * s;
        const bool ok = mbar_wait_bounded(bar, (it >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
        unsigned char* sb = smem + s * kBatchStageBytes;
        const InstanceDesc& d = *reinterpret_cast<const InstanceDesc*>(sb + kBatchDescOff);
        const StageHdr& h = *reinterpret_cast<const StageHdr*>(sb + kBatchHdrOff);
        const TileInfo& ti = *reinterpret_cast<const TileInfo*>(sb + kBatchInfoOff);
        if (ti.slot != run_slot) {
            flush();
            run_slot = ti.slot;
            run_tile = t;
            run_ctl = d.ctl;
            run_live = h.live != 0;
        }
        constexpr bool patch = PATCH;
        const PatchArrays* pe = &d.pa;
        float fo[24];
        int64_t e = 0;
#pragma unroll 1
        for (int k = 0; k < EPT; ++k) {
            const int li = tid + k * NT;
            e = static_cast<int64_t>(ti.base) + li;
            if (run_live && e < d.E.ne) {
#if ENSC_BATCH_DESC_MODE == 1
                // the instance's arrays and constants, read from the stage once:
                // the body's stores could alias the stage as far as the compiler
                // knows, so references into it would be re-read after each store
                const ElemArrays E = d.E;
                const NodeArrays N = d.N;
                const Material M = d.M;
#elif ENSC_BATCH_DESC_MODE == 2
                // arrays copied to registers, material constants read at use
                const ElemArrays E = d.E;
                const NodeArrays N = d.N;
                const Material& M = d.M;
#else
                const ElemArrays& E = d.E;
                const NodeArrays& N = d.N;
                const Material& M = d.M;
#endif
                const double dt1d = h.dt1;
                const float dt1 = static_cast<float>(dt1d);
                const float* st = reinterpret_cast<const float*>(sb);
                const MixedSrc S{reinterpret_cast<const uint32_t*>(st),
                                 st + 8 * kStageTile,
                                 reinterpret_cast<const double*>(sb + kStageV0Off),
                                 st + 44 * kStageTile,
                                 st + 26 * kStageTile,
                                 st + 32 * kStageTile,
                                 st + 45 * kStageTile,
                                 kStageTile,
                                 li};
                double d1, l1;
                element_body_mixed<true, false, true, ENSC_BATCH_MIXED_PREFETCH, true>(E, N, M, S, dt1, dt1d, e, d1, l1,
                                                                                      ei, eh, ev, bad, fo);
                dts = fmin(dts, d1);
                len = fmin(len, l1);
                if (!patch) {
                    // slot assembly: the forces to the instance's force array
                    float* __restrict__ fe = static_cast<float*>(E.fe);
                    const int64_t np = N.nn_pad, ep = E.ne_pad;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const uint32_t nj = S.conn[j * kStageTile + li];
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            if (E.slot_major) fe[(3 * j + i) * np + nj] = fo[8 * i + j];
                            else fe[(3 * j + i) * ep + e] = fo[8 * i + j];
                        }
                    }
                }
            }
        }
        if (patch && run_live) {
            // the tile's patch: its forces summed per patch node (see
            // k_element_mixed_patch); the stage's element rows hold them
            const PatchArrays PE = *pe;
            const int64_t ne = d.E.ne;
            __syncthreads();  // the stage's inputs are consumed
            float* sf = reinterpret_cast<float*>(sb);
            if (e < ne) {
#pragma unroll
                for (int i = 0; i < 24; ++i) sf[i * kStageTile + tid] = fo[i];
            }
            __syncthreads();
            patch_partials(PE, sf, static_cast<int64_t>(ti.base) / kPatchElems, tid);
        }
        __syncthreads();  // the block is done with stage s
        const int64_t tn = t + 2 * gstride;
        if (wid == 0 && tn < ntiles) {
            const ETileSrc src = *reinterpret_cast<const ETileSrc*>(sb + kBatchNextOff);
            batch_stage_issue(T, src, tn + 2 * gstride, ntiles, sb, stage0 + s * kBatchStageBytes, bar, lane);
        }
    }
    if (!timed_out) {
        flush();
    } else if (tid == 0) {
        // record the failure on the instance whose tile could not be read and
        // let the copies this block started land (bounded) before exiting
        atomicOr(&T.desc[T.etile_inst[t]].ctl->status, ST_TIMEOUT);
        for (int k = 0; k < 2; ++k) {
            const int itk = it + k;
            if (blockIdx.x + itk * gstride < ntiles) mbar_wait_bounded(bar0 + 8 * (itk & 1), (itk >> 1) & 1);
        }
    }
    element_pass_done(T);
}

// One warp per node tile.  The tile's instance slot and first node are read
// two tiles ahead and its NodeView and NodeParam lines prefetched into L1 one
// tile ahead, so a tile starts on its node rows without waiting on the
// tables.
// NT threads per block (a tuning choice: the warps are independent).
template <int NT, bool PATCH>
__global__ void __launch_bounds__(NT, ENSC_NODE_BATCH_MINB_MIXED * kNodeThreads / NT) k_node_batch_mixed(BatchTables T) {
    constexpr int W = kNodeGroupBatchMixed;
    const int lane = threadIdx.x & 31;
    const int warp = static_cast<int>((static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int nwarps = static_cast<int>((static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5);
    const int ntiles = T.counts[1];
    int slot = warp < ntiles ? __ldg(T.ntile_inst + warp) : 0;
    int slot_n = warp + nwarps < ntiles ? __ldg(T.ntile_inst + warp + nwarps) : 0;
    int base = warp < ntiles ? __ldg(T.ntile_base + warp) : 0;
    int base_n = warp + nwarps < ntiles ? __ldg(T.ntile_base + warp + nwarps) : 0;
    for (int t = warp; t < ntiles; t += nwarps) {
        const int t2 = t + 2 * nwarps;
        const int slot_nn = t2 < ntiles ? __ldg(T.ntile_inst + t2) : 0;
        const int base_nn = t2 < ntiles ? __ldg(T.ntile_base + t2) : 0;
        if (lane == 0) {
            prefetch_l1(T.nview + slot_n);
            prefetch_l1(T.nparam + slot_n);
        }
        const NodeParam p = ld_param(T.nparam + slot);
        if (p.live) {
            const NodeView v = ld_view(T.nview + slot);
            const double dt_i = p.dt_i, dt_i_1 = p.dt_i_1, amp = p.amp;
            double kin = 0.0, wext = 0.0;
            int32_t bad = 0;
            const int64_t n0 = static_cast<int64_t>(base) + static_cast<int64_t>(lane) * W;
            if (n0 < v.nn) {
                if (PATCH) {
                    node_group_mixed<W, true>(v, dt_i, dt_i_1, amp, n0, kin, wext, bad);
                } else if (v.grouped) {
                    node_group_mixed<W, false>(v, dt_i, dt_i_1, amp, n0, kin, wext, bad);
                } else {
                    const InstanceDesc& d = T.desc[slot];
                    for (int j = 0; j < W && n0 + j < v.nn; ++j)
                        node_body_mixed(d.E, d.N, d.M, dt_i, dt_i_1, amp, n0 + j, kin, wext, bad);
                }
            }
            kin = warp_sum_b(kin);
            wext = warp_sum_b(wext);
            bad = static_cast<int32_t>(__reduce_or_sync(0xffffffffu, static_cast<unsigned>(bad)));
            if (lane == 0) {
                double* part = T.ntile_part + 2 * static_cast<int64_t>(t);
                if (bad) atomicOr(&v.ctl->status, bad);
                part[0] = kin;
                atomicAdd(part + 1, wext);  // one writer per slot and pass
            }
        }
        slot = slot_n;
        slot_n = slot_nn;
        base = base_n;
        base_n = base_nn;
    }
}

}  // namespace

void launch_element_mixed(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl, const Partials& P,
                          int grid, bool init, cudaStream_t st, const PatchArrays& PA) {
    if (PA.pf) {
        if (M.plastic) {
            if (init) k_element_mixed_patch<true, true><<<grid, kStageTile, kStageSmem, st>>>(E, N, M, ctl, P, PA);
            else k_element_mixed_patch<true, false><<<grid, kStageTile, kStageSmem, st>>>(E, N, M, ctl, P, PA);
        } else {
            if (init) k_element_mixed_patch<false, true><<<grid, kStageTile, kStageSmem, st>>>(E, N, M, ctl, P, PA);
            else k_element_mixed_patch<false, false><<<grid, kStageTile, kStageSmem, st>>>(E, N, M, ctl, P, PA);
        }
        return;
    }
    if (ENSC_STAGED_MIXED && !init && E.tiles_aligned) {
        if (M.plastic) k_element_mixed_staged<true><<<grid, kStageTile, kStageSmem, st>>>(E, N, M, ctl, P);
        else k_element_mixed_staged<false><<<grid, kStageTile, kStageSmem, st>>>(E, N, M, ctl, P);
        return;
    }
    if (M.plastic) {
        if (init) k_element_mixed<true, true><<<grid, kElemThreads, 0, st>>>(E, N, M, ctl, P);
        else k_element_mixed<true, false><<<grid, kElemThreads, 0, st>>>(E, N, M, ctl, P);
    } else {
        if (init) k_element_mixed<false, true><<<grid, kElemThreads, 0, st>>>(E, N, M, ctl, P);
        else k_element_mixed<false, false><<<grid, kElemThreads, 0, st>>>(E, N, M, ctl, P);
    }
}

void launch_acceleration_mixed(const ElemArrays& E, const NodeArrays& N, const Material& M, const Ctl* ctl,
                               double* a_aos, cudaStream_t st, const PatchArrays& PA) {
    const int64_t g = (N.nn + kNodeThreads - 1) / kNodeThreads;
    k_acceleration_mixed<<<static_cast<int>(g < 65535 ? g : 65535), kNodeThreads, 0, st>>>(PA, E, N, M, ctl, a_aos);
}

void launch_node_mixed(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl, const Partials& P,
                       int grid, cudaStream_t st, const PatchArrays& PA) {
    if (PA.pf) k_node_mixed<true><<<grid, kNodeThreads, 0, st>>>(E, N, M, ctl, P, PA);
    else k_node_mixed<false><<<grid, kNodeThreads, 0, st>>>(E, N, M, ctl, P, PA);
}

// The staged passes need more than the default 48 KB of dynamic shared
// memory; the attribute is set on the current device before any launch or
// capture.
void set_element_mixed_attributes() {
    cudaFuncSetAttribute(k_element_mixed_staged<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kStageSmem));
    cudaFuncSetAttribute(k_element_mixed_staged<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kStageSmem));
    cudaFuncSetAttribute(k_element_mixed_patch<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kStageSmem));
    cudaFuncSetAttribute(k_element_mixed_patch<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kStageSmem));
    cudaFuncSetAttribute(k_element_mixed_patch<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kStageSmem));
    cudaFuncSetAttribute(k_element_mixed_patch<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kStageSmem));
}

int occupancy_element_mixed(bool plastic) {
    int nb = 0;
    set_element_mixed_attributes();
    if (ENSC_STAGED_MIXED) {
        // the staged pass needs more than the default 48 KB of dynamic shared
        // memory; the attribute is set here, on the current device, before
        // any launch or capture
        cudaFuncSetAttribute(k_element_mixed_staged<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kStageSmem));
        cudaFuncSetAttribute(k_element_mixed_staged<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kStageSmem));
        if (plastic)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_mixed_staged<true>, kStageTile, kStageSmem);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_mixed_staged<false>, kStageTile, kStageSmem);
        return nb;
    }
    if (plastic) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_mixed<true, false>, kElemThreads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_mixed<false, false>, kElemThreads, 0);
    return nb;
}

int occupancy_node_mixed() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_node_mixed<false>, kNodeThreads, 0);
    return nb;
}


void launch_element_batch_mixed(const BatchTables& T, int grid, int ept, bool patch, cudaStream_t st) {
    if (patch) k_element_batch_mixed<1, true><<<grid, kStageTile, kBatchStageSmem, st>>>(T);
    else if (ept == 2) k_element_batch_mixed<2, false><<<grid, kStageTile / 2, kBatchStageSmem, st>>>(T);
    else k_element_batch_mixed<1, false><<<grid, kStageTile, kBatchStageSmem, st>>>(T);
}
void launch_node_batch_mixed(const BatchTables& T, int grid, int threads, bool patch, cudaStream_t st) {
    if (patch) {
        if (threads == kNodeThreads / 2) k_node_batch_mixed<kNodeThreads / 2, true><<<grid, threads, 0, st>>>(T);
        else k_node_batch_mixed<kNodeThreads, true><<<grid, kNodeThreads, 0, st>>>(T);
    } else {
        if (threads == kNodeThreads / 2) k_node_batch_mixed<kNodeThreads / 2, false><<<grid, threads, 0, st>>>(T);
        else k_node_batch_mixed<kNodeThreads, false><<<grid, kNodeThreads, 0, st>>>(T);
    }
}
int occupancy_element_batch_mixed(int ept) {
    int nb = 0;
    set_element_mixed_attributes();  // the batch's init passes run the single-instance kernels
    // dynamic shared memory above the default 48 KB: set on the current
    // device before any launch or capture
    cudaFuncSetAttribute(k_element_batch_mixed<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kBatchStageSmem));
    cudaFuncSetAttribute(k_element_batch_mixed<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kBatchStageSmem));
    cudaFuncSetAttribute(k_element_batch_mixed<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kBatchStageSmem));
    if (ept == 2)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_batch_mixed<2, false>, kStageTile / 2,
                                                      kBatchStageSmem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_batch_mixed<1, false>, kStageTile, kBatchStageSmem);
    return nb;
}

int batch_element_tile(bool mixed_precision) { return mixed_precision ? kStageTile : batch_element_tile_fp64(); }
int batch_node_tile(bool mixed_precision) { return 32 * (mixed_precision ? kNodeGroupBatchMixed : kNodeGroupFp64); }
int occupancy_node_batch_mixed(int threads) {
    int nb = 0;
    if (threads == kNodeThreads / 2)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_node_batch_mixed<kNodeThreads / 2, false>, threads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_node_batch_mixed<kNodeThreads, false>, kNodeThreads, 0);
    return nb;
}

}  // namespace ensc
