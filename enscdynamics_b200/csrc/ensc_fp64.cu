// Plain FP64 stepper kernels.  Compiled with -fmad=false: every product and
// sum below is rounded separately, in the order written, which is the order
// the reference evaluates it (cited per block), so results match the
// reference CPU stepper to round-off and the CPU restatement bit-for-bit.
//
// One cycle (exDyna3D::run loop body, Explicit3D/source/exDyna3D.cpp:86-100)
// is the kernel sequence
//   between  -> [edge_prepass -> begin_exact] -> element -> node
// launched inside a CUDA graph; see ensc_capi.cu for the orchestration.
#include "ensc_device.cuh"
#include "ensc_kernels.h"
#include "ensc_stage.cuh"

#include <algorithm>
#include <cfloat>

namespace ensc {
namespace {

__device__ __forceinline__ double det3(const double m[3][3]) {
    // Eigen 3.4 bruteforce_det3_helper form (Eigen/src/LU/Determinant.h),
    // as used by all_F[e].determinant() (exDyna3D.cpp:869).
    const double h0 = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]);
    const double h1 = m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    const double h2 = m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    return (h0 - h1) + h2;
}

__device__ __forceinline__ double cof3(const double m[3][3], int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m[i1][j1] * m[i2][j2] - m[i1][j2] * m[i2][j1];
}

__device__ __forceinline__ void inv3(const double m[3][3], double r[3][3]) {
    // Eigen 3.4 compute_inverse<...,3> (Eigen/src/LU/InverseImpl.h), as used
    // by all_F[e].inverse() (exDyna3D.cpp:874).
    const double c0 = cof3(m, 0, 0), c1 = cof3(m, 1, 0), c2 = cof3(m, 2, 0);
    const double det = (c0 * m[0][0] + c1 * m[1][0]) + c2 * m[2][0];
    const double invdet = 1.0 / det;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r[i][j] = cof3(m, j, i) * invdet;
}

// Hourglass base vectors Gamma (exDyna3D.cpp:1003-1008) as signs.
__device__ __forceinline__ constexpr int tau_sign(int k, int j) {
    constexpr int T[4][8] = {{1, -1, 1, -1, 1, -1, 1, -1},
                             {-1, -1, 1, 1, 1, 1, -1, -1},
                             {-1, 1, 1, -1, 1, -1, -1, 1},
                             {-1, 1, -1, 1, 1, -1, 1, -1}};
    return T[k][j];
}

// Gamma row k as a bit mask: bit j set where the entry is +1.
__device__ __forceinline__ double tau_of(int k, int j) {
    constexpr unsigned kMask = 0x55u | (0x3Cu << 8) | (0x96u << 16) | (0x5Au << 24);
    return ((kMask >> (8 * k + j)) & 1u) ? 1.0 : -1.0;
}

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-shape block reduction (warp butterflies, then warp 0 over the
// warp results): deterministic for a given block size.
// Block sum of NV values into out_slots[i * stride + slot]; values whose bit
// is set in ACC are added to the slot (it accumulates over cycles, one writer
// per slot and pass), the others stored.
template <int NT, int NV, unsigned ACC = 0u>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* out_slots, int stride, int slot) {
    __shared__ double red[NV][NT / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double s = warp_sum(v[i]);
        if (lane == 0) red[i][wid] = s;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = lane < NT / 32 ? red[i][lane] : 0.0;
            s = warp_sum(s);
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
__device__ __forceinline__ void block_min2(double a, double b, unsigned long long* ga, unsigned long long* gb) {
    __shared__ unsigned long long ra[NT / 32], rb[NT / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long x = warp_min(ord_bits(a)), y = warp_min(ord_bits(b));
    if (lane == 0) {
        ra[wid] = x;
        rb[wid] = y;
    }
    __syncthreads();
    if (wid == 0) {
        x = lane < NT / 32 ? ra[lane] : kInfBits;
        y = lane < NT / 32 ? rb[lane] : kInfBits;
        x = warp_min(x);
        y = warp_min(y);
        if (lane == 0) {
            if (ga) atomicMin(ga, x);
            if (gb) atomicMin(gb, y);
        }
    }
    __syncthreads();
}

// Where one element's inputs are read from: rows of `stride` entries with the
// element at `i` (the instance's global arrays, or a shared-memory stage
// holding a tile of them); B0^T has its own rows so that it can stay in
// global memory while the rest is staged.
struct Fp64Src {
    const uint32_t* conn;   // [8] rows
    const double* sig;      // [6] rows
    const double* qia;      // [12] rows
    const double* vol0;
    const double* cb;       // cbrt(V0)
    const double* cb2;      // cbrt(V0^2)
    const double* eps;
    int64_t stride, i;
    const double* bt;       // [24] rows
    int64_t bt_stride, bt_i;
};

__device__ __forceinline__ Fp64Src fp64_src_global(const ElemArrays& E, int64_t e) {
    return Fp64Src{E.conn, static_cast<const double*>(E.sigma), static_cast<const double*>(E.qia), E.vol0,
                   E.cbrt_v0, E.cbrt_v0sq, static_cast<const double*>(E.eps_p), E.ne_pad, e,
                   static_cast<const double*>(E.bt), E.ne_pad, e};
}

// One element of the FP64 element pass (the kernel comment below has the
// reference mapping), shared by the single-instance, staged and batched
// kernels; inputs come from S, outputs go to the instance's arrays at
// element e.  SMEM / BT_SMEM: S's rows / B0^T rows
// are in shared memory.  PF: node rows the body reads later are prefetched
// into L1 once the connectivity is known (bit 0 the velocities, bit 1 the
// displacements).
template <bool PLASTIC, bool INIT, bool SMEM = false, bool BT_SMEM = false, int PF = 0>
__device__ __forceinline__ void element_body(const ElemArrays& E, const NodeArrays& N, const Material& M,
                                             const Fp64Src& S, const double dt1, const int64_t e, double& dts,
                                             double& len, double& e_int, double& e_hg, double& e_vis,
                                             int32_t& bad) {
    const int64_t ss = S.stride, si = S.i, bs = S.bt_stride;
    const int64_t ep = E.ne_pad, np = N.nn_pad;
    double* sig = static_cast<double*>(E.sigma);
    double* qia = static_cast<double*>(E.qia);
    double* epsp = static_cast<double*>(E.eps_p);
    double* __restrict__ fe = static_cast<double*>(E.fe);
    const double* __restrict__ X = N.x;
    const double* __restrict__ U = N.u;
    const double* __restrict__ V = static_cast<const double*>(N.v);
    const double G = M.G, lam = M.lambda;

    const double* bte = S.bt + S.bt_i;
    uint32_t n[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) n[k] = ldin<SMEM>(S.conn + k * ss + si);
    if (PF & 1) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) prefetch_l1(V + r * np + n[k]);
    }
    if (PF & 2) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) prefetch_l1(U + r * np + n[k]);
    }
    // current coordinates: hourglass projections TAU x (exact, the
    // Gamma entries are +-1) and the minimum edge (min_ele_edge :1173-1220)
    double TX[4][3];
    {
        double xyz[8][3];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            xyz[k][0] = X[n[k]];
            xyz[k][1] = X[np + n[k]];
            xyz[k][2] = X[2 * np + n[k]];
        }
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double t = tau_sign(kk, 0) > 0 ? xyz[0][c] : -xyz[0][c];
#pragma unroll
                for (int j = 1; j < 8; ++j) t = tau_sign(kk, j) > 0 ? t + xyz[j][c] : t - xyz[j][c];
                TX[kk][c] = t;
            }
        constexpr int A0[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
        constexpr int A1[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
        double m = DBL_MAX;
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const double dx = xyz[A1[k]][0] - xyz[A0[k]][0];
            const double dy = xyz[A1[k]][1] - xyz[A0[k]][1];
            const double dz = xyz[A1[k]][2] - xyz[A0[k]][2];
            const double t = __fma_rn(dz, dz, __fma_rn(dy, dy, dx * dx));
            m = t < m ? t : m;
        }
        len = sqrt(m);
    }
    // F = I + u_e B0^T (:862-865)
    double F[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
#pragma unroll kNodeUnrollFp64
    for (int k = 0; k < 8; ++k) {
        const uint32_t nk = ldin<SMEM>(S.conn + k * ss + si);
        const double uu[3] = {U[nk], U[np + nk], U[2 * np + nk]};
        const double* bk = bte + 3 * k * bs;
        const double bb[3] = {ldin<BT_SMEM>(bk), ldin<BT_SMEM>(bk + bs), ldin<BT_SMEM>(bk + 2 * bs)};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) F[r][c] = __fma_rn(uu[r], bb[c], F[r][c]);
    }
    F[0][0] = 1.0 + F[0][0];
    F[1][1] = 1.0 + F[1][1];
    F[2][2] = 1.0 + F[2][2];
    const double J = det3(F);
    double Fi[3][3];
    inv3(F, Fi);
    if (!(J > 0.0)) bad |= ST_INVERTED;
    // per node: L0 = v_e B0^T, VT = v_e Gamma^T (signed sums), NX2 (:1024)
    double L0[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    double VT[3][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
    double nx2 = 0.0;
#pragma unroll kNodeUnrollFp64
    for (int j = 0; j < 8; ++j) {
        const uint32_t nj = ldin<SMEM>(S.conn + j * ss + si);
        const double* bk = bte + 3 * j * bs;
        const double bb[3] = {ldin<BT_SMEM>(bk), ldin<BT_SMEM>(bk + bs), ldin<BT_SMEM>(bk + 2 * bs)};
        const double vj[3] = {V[nj], V[np + nj], V[2 * np + nj]};
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int c = 0; c < 3; ++c) L0[r][c] = __fma_rn(vj[r], bb[c], L0[r][c]);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) VT[r][kk] = tau_of(kk, j) > 0.0 ? VT[r][kk] + vj[r] : VT[r][kk] - vj[r];
        }
        nx2 = nx2 + __fma_rn(bb[2], bb[2], __fma_rn(bb[1], bb[1], bb[0] * bb[0]));
    }
    // L = L0 F^-1 (= v_e b^T, :928); HIA = VT - L0 TX^T (= v_e ATAU^T, :1020-1021)
    double L[3][3], HIA[3][4];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
            L[r][c] = __fma_rn(L0[r][2], Fi[2][c], __fma_rn(L0[r][1], Fi[1][c], L0[r][0] * Fi[0][c]));
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
            HIA[r][kk] = VT[r][kk] - __fma_rn(L0[r][2], TX[kk][2], __fma_rn(L0[r][1], TX[kk][1], L0[r][0] * TX[kk][0]));
    }
    const double vr = (L[0][0] + L[1][1]) + L[2][2];
    // Jaumann stress update (:930-973)
    double eps[6];
    eps[0] = L[0][0] * dt1;
    eps[1] = L[1][1] * dt1;
    eps[2] = L[2][2] * dt1;
    eps[3] = (L[0][1] + L[1][0]) / 2.0 * dt1;
    eps[4] = (L[0][2] + L[2][0]) / 2.0 * dt1;
    eps[5] = (L[1][2] + L[2][1]) / 2.0 * dt1;
    const double w0 = (L[0][1] - L[1][0]) / 2.0;
    const double w1 = (L[0][2] - L[2][0]) / 2.0;
    const double w2 = (L[1][2] - L[2][1]) / 2.0;
    const double tr = (eps[0] + eps[1]) + eps[2];
    double s[6], so[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) so[i] = S.sig[i * ss + si];
    double inc[6];
    inc[0] = (lam * tr + 2.0 * G * eps[0]) + 2.0 * so[3] * w0 * dt1 + 2.0 * so[4] * w1 * dt1;
    inc[1] = (lam * tr + 2.0 * G * eps[1]) - 2.0 * so[3] * w0 * dt1 + 2.0 * so[5] * w2 * dt1;
    inc[2] = (lam * tr + 2.0 * G * eps[2]) - 2.0 * so[4] * w1 * dt1 - 2.0 * so[5] * w2 * dt1;
    inc[3] = (2.0 * G * eps[3]) + (so[1] - so[0]) * w0 * dt1 + so[5] * w1 * dt1;
    inc[4] = (2.0 * G * eps[4]) + (so[2] - so[0]) * w1 * dt1 + so[5] * w0 * dt1;
    inc[5] = (2.0 * G * eps[5]) + (so[2] - so[1]) * w2 * dt1 + so[3] * w1 * dt1 - so[4] * w0 * dt1;
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = so[i] + inc[i];
    if (PLASTIC) {
        // J2 radial return, linear isotropic hardening (no reference
        // counterpart; the elastic instantiation omits it).
        const double pm = ((s[0] + s[1]) + s[2]) / 3.0;
        const double d0 = s[0] - pm, d1 = s[1] - pm, d2 = s[2] - pm;
        const double j2 = 0.5 * ((d0 * d0 + d1 * d1) + d2 * d2) + ((s[3] * s[3] + s[4] * s[4]) + s[5] * s[5]);
        const double seq = sqrt(3.0 * j2);
        const double ep_old = S.eps[si];
        const double sy = M.yield0 + M.hardening * ep_old;
        if (seq > sy) {
            const double dl = (seq - sy) / (3.0 * G + M.hardening);
            const double r = 1.0 - 3.0 * G * dl / seq;
            s[0] = d0 * r + pm;
            s[1] = d1 * r + pm;
            s[2] = d2 * r + pm;
            s[3] = s[3] * r;
            s[4] = s[4] * r;
            s[5] = s[5] * r;
            if (!INIT) epsp[e] = ep_old + dl;
        }
    }
    if (!INIT) {
#pragma unroll
        for (int i = 0; i < 6; ++i) sig[i * ep + e] = s[i];
    }
    const double V0 = S.vol0[si];
    const double Vc = J * V0;
    {
        double w = 0.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const double sm = 0.5 * (so[i] + s[i]);
            w = w + (i < 3 ? 1.0 : 2.0) * sm * eps[i];
        }
        e_int += w * Vc;
    }
    // hourglass coefficients and history (:1038-1050); Gq = QIA + CR HIA
    const double r43 = 4.0 / 3.0;
    const double r1s8 = 1.0 / sqrt(8.0);
    const double DR = M.c_dr * (r43 * G + M.K) * 0.1 * nx2 * Vc * r1s8 * dt1;
    const double CR = M.c_cr * M.rho * V0 / Vc * S.cb2[si] * M.wos / 4.0;
    double Gq[3][4];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            const double q = __fma_rn(DR, HIA[i][kk], S.qia[(4 * i + kk) * ss + si]);
            if (!INIT) qia[(4 * i + kk) * ep + e] = q;
            Gq[i][kk] = __fma_rn(CR, HIA[i][kk], q);
        }
    // bulk viscosity pressure (:1073-1109)
    const bool visc = !(fabs(vr) < 1.0e-10);
    double pv = 0.0;
    if (visc) {
        const double rho_c = M.rho / J;
        const double l0 = S.cb[si];
        const double m0 = vr < 0.0 ? vr : 0.0;
        pv = rho_c * l0 * (M.cvisq * M.cvisq * l0 * vr * m0 - M.cvisl * M.wos * vr);
        e_vis += -(pv * Vc * vr) * dt1;
    }
    // Z = Vc F^-1 (sigma - p I) - W^T, W = Gq TX
    const double Sp[3][3] = {{s[0] - pv, s[3], s[4]}, {s[3], s[1] - pv, s[5]}, {s[4], s[5], s[2] - pv}};
    double W[3][3], Z[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            W[i][c] = __fma_rn(Gq[i][3], TX[3][c],
                               __fma_rn(Gq[i][2], TX[2][c], __fma_rn(Gq[i][1], TX[1][c], Gq[i][0] * TX[0][c])));
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i)
            Z[c][i] = Vc * __fma_rn(Fi[c][2], Sp[2][i], __fma_rn(Fi[c][1], Sp[1][i], Fi[c][0] * Sp[0][i])) - W[i][c];
    // hourglass power sum_j h_j . v_j = Gq : HIA
    {
        double hp = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) hp = __fma_rn(Gq[i][kk], HIA[i][kk], hp);
        e_hg += hp * dt1;
    }
    // nodal forces f_j = -(B0_j Z) - Gamma_j Gq^T
    // (= -b_j sigma V - h_j + p b_j V: :985-997, :1070, :1106)
#pragma unroll kNodeUnrollFp64
    for (int j = 0; j < 8; ++j) {
        const double* bk = bte + 3 * j * bs;
        const double b0 = ldin<BT_SMEM>(bk), b1 = ldin<BT_SMEM>(bk + bs), b2 = ldin<BT_SMEM>(bk + 2 * bs);
        double* fej;
        int64_t fst;
        if (E.slot_major) {
            fej = fe + 3 * j * np + ldin<SMEM>(S.conn + j * ss + si);
            fst = np;
        } else {
            fej = fe + 3 * j * ep + e;
            fst = ep;
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double tg = tau_of(0, j) > 0.0 ? Gq[i][0] : -Gq[i][0];
#pragma unroll
            for (int kk = 1; kk < 4; ++kk) tg = tau_of(kk, j) > 0.0 ? tg + Gq[i][kk] : tg - Gq[i][kk];
            fej[i * fst] = -__fma_rn(b2, Z[2][i], __fma_rn(b1, Z[1][i], b0 * Z[0][i])) - tg;
        }
    }
    // compute_dtStable (:828-834)
    {
        const double cd = M.wos;
        const double m0 = vr < 0.0 ? vr : 0.0;
        const double xi = M.cvisl - M.cvisq * M.cvisq * len / cd * m0;
        dts = (sqrt(1.0 + xi * xi) - xi) * len / cd;
    }
    if (!isfinite(dts)) bad |= ST_NONFINITE;
}

// Element pass: add_inForce_to_rhs's element loop body
// (exDyna3D.cpp:556-573): kinematics, Jaumann stress (+ J2 return),
// hourglass, bulk viscosity, element dt and min edge.  Writes the element's
// 8x3 nodal forces to fe for the node-centric gather.
//
// Register-lean structure: the element's nodes are streamed once for the
// kinematics (b^T, L, hourglass vectors, HIA) and once more for the forces;
// per-node rows of b^T and ATAU are recomputed from B0^T (L1-resident) rather
// than held, so no 8x3 / 4x8 array stays live.  Every value is the same
// expression, in the same order, as the CPU restatement (explicit fma only).
template <bool PLASTIC, bool INIT>
__global__ void __launch_bounds__(kElemThreads, ENSC_ELEM_MINB_FP64) k_element(ElemArrays E, NodeArrays N, Material M, Ctl* ctl,
                                                             Partials P) {
    if (ctl->done) return;
    const double dt1 = INIT ? 0.0 : ctl->dt_i_1;
    const int64_t ne = E.ne;
    double e_int = 0.0, e_hg = 0.0, e_vis = 0.0;
    double dts_min = DBL_MAX, len_min = DBL_MAX;
    int32_t bad = 0;

    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t e_end = (ne + blockDim.x - 1) / blockDim.x * blockDim.x;
    for (int64_t e0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e0 < e_end; e0 += stride) {
        const bool live = e0 < ne;
        const int64_t e = live ? e0 : 0;
        double dts = DBL_MAX, len = DBL_MAX;
        if (live) element_body<PLASTIC, INIT>(E, N, M, fp64_src_global(E, e), dt1, e, dts, len, e_int, e_hg, e_vis, bad);
        dts_min = dts < dts_min ? dts : dts_min;
        len_min = len < len_min ? len : len_min;
    }
    if (bad) atomicOr(&ctl->status, bad);
    block_min2<kElemThreads>(dts_min, len_min, &ctl->dts_next, &ctl->len_min);
    if (!INIT) {
        double v3[3] = {e_int, e_hg, e_vis};
        block_sum<kElemThreads, 3, 7u>(v3, P.elem, P.n_elem_blocks, blockIdx.x);
    }
}

// One node of the node pass (see the kernel comment below); shared by the
// single-instance and batched kernels.
__device__ __forceinline__ void node_body(const ElemArrays& E, const NodeArrays& N, const Material& M,
                                          const double dt_i, const double dt_i_1, const double amp, const int64_t n, double& kin,
                                          double& wext, int32_t& bad) {
    const int64_t np = N.nn_pad, ep = E.ne_pad;
    const double* __restrict__ fe = static_cast<const double*>(E.fe);
    double* __restrict__ V = static_cast<double*>(N.v);
    const double half = (dt_i + dt_i_1);
    const double dt_avg = (dt_i + dt_i_1) / 2.0;

    double f[3];
    if (E.slot_major) {
        // the reference's ((((((a0+a1)+a2)+a3)+a4)+a5)+a6)+a7 over the
        // slots that hold an element (an absent slot adds +0.0)
        f[0] = f[1] = f[2] = 0.0;
        const uint32_t msk = N.slot_mask[n];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if ((msk >> k) & 1u) {
#pragma unroll
                for (int c = 0; c < 3; ++c) f[c] = f[c] + fe[(3 * k + c) * np + n];
            }
        }
    } else if (N.csr_ptr == nullptr) {
        f[0] = f[1] = f[2] = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t el = __ldg(N.ell + k * np + n);
            if (el != ENSC_NONE) {
#pragma unroll
                for (int c = 0; c < 3; ++c) f[c] = f[c] + fe[(3 * k + c) * ep + el];
            }
        }
    } else {
        // general lists: entries sorted by (slot, element); each slot's
        // contributions are summed first (the reference's per-slot +=
        // in element order), then added to the running total
        f[0] = f[1] = f[2] = 0.0;
        const int64_t b = N.csr_ptr[n], t = N.csr_ptr[n + 1];
        int cur = -1;
        double sl[3] = {0.0, 0.0, 0.0};
        for (int64_t i = b; i < t; ++i) {
            const uint32_t ent = N.csr_ent[i];
            const int k = static_cast<int>(ent & 7u);
            const uint32_t el = ent >> 3;
            if (k != cur) {
                if (cur >= 0) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) f[c] = f[c] + sl[c];
                }
                cur = k;
#pragma unroll
                for (int c = 0; c < 3; ++c) sl[c] = 0.0 + fe[(3 * k + c) * ep + el];
            } else {
#pragma unroll
                for (int c = 0; c < 3; ++c) sl[c] = sl[c] + fe[(3 * k + c) * ep + el];
            }
        }
        if (cur >= 0) {
#pragma unroll
            for (int c = 0; c < 3; ++c) f[c] = f[c] + sl[c];
        }
    }
    const double im = N.inv_mass[n];
    const uint32_t code = N.bc[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double a = f[c];
        double g = 0.0;
        if (M.gravity_on) {
            g = amp * M.gravity_value * M.gravity_dir[c] / im;  // apply_gravity (:809-824)
            a = a + g;
        }
        const uint32_t cc = (code >> (2 * c)) & 3u;
        double r = 0.0, rf = 0.0;
        if (cc & 2u) {
            r = -a;
            a = 0.0;
        }
        if ((cc & 1u) && a != 0.0) {
            rf = -a;
            r = -a;
            a = 0.0;
        }
        if (cc) N.rf[c * np + n] = rf;
        a = a * im;
        const double vo = V[c * np + n];
        const double vn = vo + half * a / 2.0;
        V[c * np + n] = vn;
        N.u[c * np + n] = N.u[c * np + n] + dt_i * vn;
        N.x[c * np + n] = N.x[c * np + n] + dt_i * vn;
        const double vb = 0.5 * (vo + vn);
        wext = wext + (g + r) * dt_avg * vb;
        kin = kin + 0.5 * (vn * vn) / im;
        if (!isfinite(vn)) bad |= ST_NONFINITE;
    }
}

// ---- staged element pass ------------------------------------------------
// As k_element, with each block walking tiles of kStageTileF64 consecutive
// elements whose streamed inputs -- connectivity, sigma, QIA, V0, cbrt(V0),
// cbrt(V0^2), eps_p and, when BT, B0^T -- thread 0 copies into one of two
// shared-memory stages with bulk copies one tile ahead of the compute.  The
// arithmetic is element_body's, so results are bit-identical to k_element.
constexpr int kStageTileF64 = ENSC_STAGE_TILE_FP64;
// resident blocks per SM of the staged FP64 passes (same threads per SM for
// any tile size)
constexpr int kStageMinbF64 = 256 / kStageTileF64;
constexpr int kF64StageRows = 22;  // double rows before B0^T: 6 sigma, 12 QIA, V0, cbrt V0, cbrt V0^2, eps_p
template <bool BT>
constexpr uint32_t f64_stage_bytes() {
    return 8u * kStageTileF64 * 4u + static_cast<uint32_t>(kF64StageRows + (BT ? 24 : 0)) * kStageTileF64 * 8u;
}
template <bool BT>
constexpr size_t f64_stage_smem() {
    return 2 * static_cast<size_t>(f64_stage_bytes<BT>()) + 16;
}

// double row r of the stage in global memory
__device__ __forceinline__ const double* f64_stage_row(const ElemArrays& E, int r) {
    const int64_t ep = E.ne_pad;
    if (r < 6) return static_cast<const double*>(E.sigma) + r * ep;
    if (r < 18) return static_cast<const double*>(E.qia) + (r - 6) * ep;
    if (r == 18) return E.vol0;
    if (r == 19) return E.cbrt_v0;
    if (r == 20) return E.cbrt_v0sq;
    if (r == 21) return static_cast<const double*>(E.eps_p);
    return static_cast<const double*>(E.bt) + (r - kF64StageRows) * ep;
}

// Warp 0: the tile starting at element `base` into the stage at shared
// address dst, completing on bar (rows padded to 32 entries and 256-byte
// aligned: every copy is 16-byte aligned and a multiple of 128 bytes); lane
// 0 arms the barrier, then the lanes start the row copies between them.
__device__ __forceinline__ uint32_t f64_stage_count(const ElemArrays& E, int64_t base) {
    const int64_t left = E.ne_pad - base;
    return static_cast<uint32_t>(left < kStageTileF64 ? left : kStageTileF64);
}
template <bool PLASTIC, bool BT>
__device__ __forceinline__ uint32_t f64_stage_tx_bytes(uint32_t cnt) {
    constexpr int drows = kF64StageRows + (BT ? 24 : 0);
    constexpr int dcopies = PLASTIC ? drows : drows - 1;
    return 8u * cnt * 4u + static_cast<uint32_t>(dcopies) * cnt * 8u;
}
template <bool PLASTIC, bool BT>
__device__ __forceinline__ void f64_stage_issue(const ElemArrays& E, uint32_t dst, uint32_t bar, int64_t base,
                                                int lane) {
    constexpr int drows = kF64StageRows + (BT ? 24 : 0);
    const uint32_t cnt = f64_stage_count(E, base);
    if (lane == 0) mbar_arrive_expect_tx(bar, f64_stage_tx_bytes<PLASTIC, BT>(cnt));
    __syncwarp();
    fence_proxy_async_smem();  // the block's reads of this stage come before the copies into it
    const uint32_t dbase = dst + 8u * kStageTileF64 * 4u;
    for (int q = lane; q < 8 + drows; q += 32) {
        if (q < 8) {
            bulk_g2s(dst + q * (kStageTileF64 * 4u), E.conn + q * E.ne_pad + base, cnt * 4u, bar);
        } else {
            const int r = q - 8;
            if (PLASTIC || r != 21)  // eps_p is read only with J2
                bulk_g2s(dbase + r * (kStageTileF64 * 8u), f64_stage_row(E, r) + base, cnt * 8u, bar);
        }
    }
}

template <bool PLASTIC, bool BT>
__global__ void __launch_bounds__(kStageTileF64, BT ? kStageMinbF64 : kStageMinbF64 * 3 / 2)
    k_element_staged(ElemArrays E, NodeArrays N, Material M, Ctl* ctl, Partials P) {
    if (ctl->done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr uint32_t SB = f64_stage_bytes<BT>();
    constexpr int T = kStageTileF64;
    const double dt1 = ctl->dt_i_1;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t stage0 = smem_addr(smem);
    const uint32_t bar0 = stage0 + 2 * SB;
    const int64_t ntiles = (E.ne + T - 1) / T;
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
            if (t < ntiles) f64_stage_issue<PLASTIC, BT>(E, stage0 + s * SB, bar0 + 8 * s, t * T, lane);
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
        const int64_t e = t * T + tid;
        if (e < E.ne) {
            const unsigned char* st = smem + s * SB;
            const double* d = reinterpret_cast<const double*>(st + 8 * T * 4);
            const Fp64Src S{reinterpret_cast<const uint32_t*>(st), d, d + 6 * T, d + 18 * T, d + 19 * T, d + 20 * T,
                            d + 21 * T, T, tid,
                            BT ? d + kF64StageRows * T : static_cast<const double*>(E.bt),
                            BT ? static_cast<int64_t>(T) : E.ne_pad, BT ? static_cast<int64_t>(tid) : e};
            double dts, len;
            element_body<PLASTIC, false, true, BT>(E, N, M, S, dt1, e, dts, len, e_int, e_hg, e_vis, bad);
            dts_min = dts < dts_min ? dts : dts_min;
            len_min = len < len_min ? len : len_min;
        }
        __syncthreads();  // the block is done with stage s
        const int64_t tn = t + 2 * gstride;
        if (wid == 0 && tn < ntiles) f64_stage_issue<PLASTIC, BT>(E, stage0 + s * SB, bar, tn * T, lane);
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
    block_min2<kStageTileF64>(dts_min, len_min, &ctl->dts_next, &ctl->len_min);
    double v3[3] = {e_int, e_hg, e_vis};
    block_sum<kStageTileF64, 3, 7u>(v3, P.elem, P.n_elem_blocks, blockIdx.x);
}

// ---- output: the last cycle's acceleration --------------------------------
// solution_a as compute_a leaves it (exDyna3D.cpp:642-644) in the last cycle
// -- assembled element forces, gravity, the acceleration boundary conditions,
// times the inverse mass -- which output_results writes (:231).  The node
// pass does not store it; this pass evaluates it again from the element
// forces that the last force pass left in fe, with the node pass's
// arithmetic in the node pass's order (the grouped layout adds all 8 slots,
// empty ones as the zeros they hold).  Writes interleaved xyz per node.
__global__ void __launch_bounds__(kNodeThreads) k_acceleration(ElemArrays E, NodeArrays N, Material M, const Ctl* ctl,
                                                               double* a_out) {
    const int64_t np = N.nn_pad, ep = E.ne_pad;
    const double* __restrict__ fe = static_cast<const double*>(E.fe);
    const bool grouped = E.slot_major && E.tiles_aligned;
    const double amp = (M.gravity_on && M.amp_n > 0) ? gravity_amplitude(M.amp, M.amp_n, ctl->time, ctl->dt_i) : 1.0;
    for (int64_t n = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; n < N.nn;
         n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double f[3] = {0.0, 0.0, 0.0};
        if (E.slot_major) {
            const uint32_t msk = grouped ? 0xffu : N.slot_mask[n];
#pragma unroll
            for (int k = 0; k < 8; ++k)
                if ((msk >> k) & 1u) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) f[c] = f[c] + fe[(3 * k + c) * np + n];
                }
        } else if (N.csr_ptr == nullptr) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t el = N.ell[k * np + n];
                if (el != ENSC_NONE) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) f[c] = f[c] + fe[(3 * k + c) * ep + el];
                }
            }
        } else {
            int cur = -1;
            double sl[3] = {0.0, 0.0, 0.0};
            for (int64_t i = N.csr_ptr[n]; i < N.csr_ptr[n + 1]; ++i) {
                const uint32_t ent = N.csr_ent[i];
                const int k = static_cast<int>(ent & 7u);
                const uint32_t el = ent >> 3;
                if (k != cur) {
                    if (cur >= 0) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) f[c] = f[c] + sl[c];
                    }
                    cur = k;
#pragma unroll
                    for (int c = 0; c < 3; ++c) sl[c] = 0.0 + fe[(3 * k + c) * ep + el];
                } else {
#pragma unroll
                    for (int c = 0; c < 3; ++c) sl[c] = sl[c] + fe[(3 * k + c) * ep + el];
                }
            }
            if (cur >= 0) {
#pragma unroll
                for (int c = 0; c < 3; ++c) f[c] = f[c] + sl[c];
            }
        }
        const double im = N.inv_mass[n];
        const uint32_t code = N.bc[n];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double a = f[c];
            if (M.gravity_on) a = a + amp * M.gravity_value * M.gravity_dir[c] / im;
            const uint32_t cc = (code >> (2 * c)) & 3u;
            if (cc & 2u) a = 0.0;
            if ((cc & 1u) && a != 0.0) a = 0.0;
            a_out[3 * n + c] = a * im;
        }
    }
}

// ---- warp-pipelined element pass ---------------------------------------
// As k_element_staged (B0^T staged too), but every warp runs its own
// pipeline over tiles of 32 consecutive elements: its own two stages, its
// own barriers, a stage reused as soon as its 32 lanes are done with it, and
// no block-wide barrier per tile.  element_body's arithmetic, so results are
// bit-identical to the other FP64 element passes.
constexpr int kF64WarpTile = 32;
// B0^T staged with the other rows (1) or read from global memory through L1
// (0, a smaller stage: more warps fit in shared memory)
constexpr bool kF64WarpBt = ENSC_F64_WARP_BT != 0;
constexpr uint32_t kF64WarpStageBytes =
    8u * kF64WarpTile * 4u + (kF64StageRows + (kF64WarpBt ? 24 : 0)) * kF64WarpTile * 8u;
constexpr int kF64PipeWarps = ENSC_F64_PIPE_WARPS;
constexpr size_t kF64WarpPipeSmem = static_cast<size_t>(kF64PipeWarps) * (2 * kF64WarpStageBytes + 16);

template <bool PLASTIC>
__device__ __forceinline__ void f64_warp_stage_issue(const ElemArrays& E, uint32_t dst, uint32_t bar, int64_t base,
                                                     int lane) {
    constexpr int drows = kF64StageRows + (kF64WarpBt ? 24 : 0);
    // whole 32-entry tiles of rows padded to multiples of 32: 128- and
    // 256-byte copies
    if (lane == 0) mbar_arrive_expect_tx(bar, f64_stage_tx_bytes<PLASTIC, kF64WarpBt>(kF64WarpTile));
    __syncwarp();
    fence_proxy_async_smem();  // the warp's reads of this stage come before the copies into it
    const uint32_t dbase = dst + 8u * kF64WarpTile * 4u;
    for (int q = lane; q < 8 + drows; q += 32) {
        if (q < 8) {
            bulk_g2s(dst + q * (kF64WarpTile * 4u), E.conn + q * E.ne_pad + base, kF64WarpTile * 4u, bar);
        } else {
            const int r = q - 8;
            if (PLASTIC || r != 21)  // eps_p is read only with J2
                bulk_g2s(dbase + r * (kF64WarpTile * 8u), f64_stage_row(E, r) + base, kF64WarpTile * 8u, bar);
        }
    }
}

template <bool PLASTIC>
__global__ void __launch_bounds__(32 * kF64PipeWarps, ENSC_F64_PIPE_MINB)
    k_element_fp64_warp(ElemArrays E, NodeArrays N, Material M, Ctl* ctl, Partials P) {
    if (ctl->done) return;
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int T = kF64WarpTile;
    const double dt1 = ctl->dt_i_1;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    unsigned char* wst = smem + static_cast<size_t>(wid) * 2 * kF64WarpStageBytes;
    const uint32_t stage0 = smem_addr(wst);
    const uint32_t bar0 = smem_addr(smem + static_cast<size_t>(kF64PipeWarps) * 2 * kF64WarpStageBytes) + 16u * wid;
    const int64_t ntiles = (E.ne + T - 1) / T;
    const int64_t wstride = static_cast<int64_t>(gridDim.x) * kF64PipeWarps;
    const int64_t w0 = static_cast<int64_t>(blockIdx.x) * kF64PipeWarps + wid;
    if (lane == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        mbar_init_fence();
    }
    __syncwarp();
    for (int s = 0; s < 2; ++s) {
        const int64_t t = w0 + s * wstride;
        if (t < ntiles) f64_warp_stage_issue<PLASTIC>(E, stage0 + s * kF64WarpStageBytes, bar0 + 8 * s, t * T, lane);
    }
    double e_int = 0.0, e_hg = 0.0, e_vis = 0.0;
    double dts_min = DBL_MAX, len_min = DBL_MAX;
    int32_t bad = 0;
    bool timed_out = false;
    int it = 0;
    for (int64_t t = w0; t < ntiles; t += wstride, ++it) {
        const int s = it & 1;
        const uint32_t bar = bar0 + 8 * s;
        const bool ok = mbar_wait_bounded(bar, (it >> 1) & 1);
        if (__any_sync(0xffffffffu, !ok)) {
            timed_out = true;
            break;
        }
        const int64_t e = t * T + lane;
        if (e < E.ne) {
            const unsigned char* st = wst + s * kF64WarpStageBytes;
            const double* d = reinterpret_cast<const double*>(st + 8 * T * 4);
            const Fp64Src S{reinterpret_cast<const uint32_t*>(st), d, d + 6 * T, d + 18 * T, d + 19 * T, d + 20 * T,
                            d + 21 * T, T, lane,
                            kF64WarpBt ? d + kF64StageRows * T : static_cast<const double*>(E.bt),
                            kF64WarpBt ? static_cast<int64_t>(T) : E.ne_pad,
                            kF64WarpBt ? static_cast<int64_t>(lane) : e};
            double dts, len;
            element_body<PLASTIC, false, true, kF64WarpBt, ENSC_F64_PREFETCH>(E, N, M, S, dt1, e, dts, len, e_int,
                                                                              e_hg, e_vis, bad);
            dts_min = dts < dts_min ? dts : dts_min;
            len_min = len < len_min ? len : len_min;
        }
        const int64_t tn = t + 2 * wstride;
        if (tn < ntiles) f64_warp_stage_issue<PLASTIC>(E, stage0 + s * kF64WarpStageBytes, bar, tn * T, lane);
    }
    if (timed_out) {
        // record the failure and let the copies this warp started land
        // (bounded) before the block's shared memory is released
        if (lane == 0) {
            atomicOr(&ctl->status, ST_TIMEOUT);
            for (int k = 0; k < 2; ++k) {
                const int itk = it + k;
                if (w0 + itk * wstride < ntiles) mbar_wait_bounded(bar0 + 8 * (itk & 1), (itk >> 1) & 1);
            }
        }
        __syncwarp();
    }
    if (bad) atomicOr(&ctl->status, bad);
    block_min2<32 * kF64PipeWarps>(dts_min, len_min, &ctl->dts_next, &ctl->len_min);
    double v3[3] = {e_int, e_hg, e_vis};
    block_sum<32 * kF64PipeWarps, 3, 7u>(v3, P.elem, P.n_elem_blocks, blockIdx.x);
}

// W consecutive nodes of the node pass with 16-byte row accesses: the same
// arithmetic per node as node_body on the slot-major layout, in the same
// order.  Slots the mask marks empty are skipped, or (ENSC_NODE_ALL_SLOTS)
// added as the zeros they hold, as the reference adds all 8 slot vectors:
// the slot-major rows start zeroed and only the slot's element writes them.
// Nodes at or past nn (row padding) are loaded and stored back unchanged.
template <int W>
__device__ __forceinline__ void node_group(const NodeView& N, const double dt_i, const double dt_i_1, const double amp,
                                           const int64_t n0, double& kin, double& wext, int32_t& bad) {
    const int64_t np = N.np, nn = N.nn;
    const double* __restrict__ fe = static_cast<const double*>(N.fe);
    double* __restrict__ V = static_cast<double*>(N.v);
    const double half = (dt_i + dt_i_1);
    const double dt_avg = (dt_i + dt_i_1) / 2.0;
    double f[3][W];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int j = 0; j < W; ++j) f[c][j] = 0.0;
    const uint32_t msk = ENSC_NODE_ALL_SLOTS ? 0xffffffffu : ld_bytes<W>(N.slot_mask + n0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        uint32_t sel = 0;
#pragma unroll
        for (int j = 0; j < W; ++j) sel |= ((msk >> (8 * j + k)) & 1u) << j;
        if (sel) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double r[W];
                ld_row<W>(fe + (3 * k + c) * np + n0, r);
#pragma unroll
                for (int j = 0; j < W; ++j)
                    if ((sel >> j) & 1u) f[c][j] = f[c][j] + r[j];
            }
        }
    }
    double im[W];
    ld_row<W>(N.inv_mass + n0, im);
    const uint32_t code = ld_bytes<W>(N.bc + n0);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double vo[W], uo[W], xo[W], vn[W], un[W], xn[W];
        ld_row<W>(V + c * np + n0, vo);
        ld_row<W>(N.u + c * np + n0, uo);
        ld_row<W>(N.x + c * np + n0, xo);
#pragma unroll
        for (int j = 0; j < W; ++j) {
            vn[j] = vo[j];
            un[j] = uo[j];
            xn[j] = xo[j];
            if (n0 + j >= nn) continue;
            double a = f[c][j];
            double g = 0.0;
            if (N.gravity_on) {
                g = amp * N.gravity_value * N.gravity_dir[c] / im[j];
                a = a + g;
            }
            const uint32_t cc = (code >> (8 * j + 2 * c)) & 3u;
            double r = 0.0, rf = 0.0;
            if (cc & 2u) {
                r = -a;
                a = 0.0;
            }
            if ((cc & 1u) && a != 0.0) {
                rf = -a;
                r = -a;
                a = 0.0;
            }
            if (cc) N.rf[c * np + n0 + j] = rf;
            a = a * im[j];
            vn[j] = vo[j] + half * a / 2.0;
            un[j] = uo[j] + dt_i * vn[j];
            xn[j] = xo[j] + dt_i * vn[j];
            const double vb = 0.5 * (vo[j] + vn[j]);
            wext = wext + (g + r) * dt_avg * vb;
            kin = kin + 0.5 * (vn[j] * vn[j]) / im[j];
            if (!isfinite(vn[j])) bad |= ST_NONFINITE;
        }
        st_row<W>(V + c * np + n0, vn);
        st_row<W>(N.u + c * np + n0, un);
        st_row<W>(N.x + c * np + n0, xn);
    }
}

// Node pass: gather of the element forces in slot order (the reference's
// ((((((a0+a1)+a2)+a3)+a4)+a5)+a6)+a7, exDyna3D.cpp:638-639), gravity
// (:819-824), boundary conditions on a (:2029-2145), a = f M^-1 (:642-644),
// v += (dt_i + dt_i_1) a / 2, u += dt_i v, x += dt_i v (:646-654, :688-696).
__global__ void __launch_bounds__(kNodeThreads, ENSC_NODE_MINB_FP64) k_node(ElemArrays E, NodeArrays N, Material M, Ctl* ctl, Partials P) {
    if (ctl->done) return;
    // stable dt of this cycle (update_minVertex_perMaterial_and_dt :673-679)
    double dt_i;
    const double dt_i_1 = ctl->dt_i_1;
    if (ctl->dt_final) {
        dt_i = ctl->dt_i;
    } else {
        const double lmin = bits_ord(ctl->len_min);
        double d = lmin / ctl->wos;
        const double tmp = ctl->dts_cur;
        d = d < tmp ? d : tmp;
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
        constexpr int W = kNodeGroupFp64;
        const NodeView nv = node_view(E, N, M, ctl);
        for (int64_t g = t0; g * W < nn; g += stride) node_group<W>(nv, dt_i, dt_i_1, amp, g * W, kin, wext, bad);
    } else {
        for (int64_t n = t0; n < nn; n += stride) node_body(E, N, M, dt_i, dt_i_1, amp, n, kin, wext, bad);
    }
    if (bad) atomicOr(&ctl->status, bad);
    double v2[2] = {kin, wext};
    block_sum<kNodeThreads, 2, 2u>(v2, P.node, P.n_node_blocks, blockIdx.x);
}


// ---- batched instances --------------------------------------------------------
// Element tiles of kStageTileF64 elements and node tiles of
// 32 * kNodeGroupFp64 nodes, each inside one instance whose arrays, material
// and control block come from the instance table.  The element pass runs the
// staged pipeline over the tile list, one tile per block at a time; the node
// pass gives each node tile to one warp.  Each tile accumulates its work terms across
// cycles (one owner per tile and pass) and keeps its latest kinetic energy;
// k_fold_batch folds them per instance in tile order, so the totals do not
// depend on scheduling.  Arithmetic per element and node is that of
// the single-instance kernels, so states are bit-identical to them.
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

// A batch stage: the element rows of a tile of kF64BatchTile elements (as the
// single-instance stage, B0^T included), then the tile's instance
// descriptor, its element-pass scalars (StageHdr), the TileInfo the filling
// warp writes, and the ETileSrc record of the tile that uses the stage next
// (as in the mixed batch pass).
constexpr int kF64BatchTile = ENSC_F64_BATCH_TILE;
static_assert(kF64BatchTile % 32 == 0, "whole warps per tile");
constexpr uint32_t kF64DescOff =
    8u * kF64BatchTile * 4u + static_cast<uint32_t>(kF64StageRows + 24) * kF64BatchTile * 8u;
constexpr uint32_t kF64HdrOff = kF64DescOff + sizeof(InstanceDesc);
constexpr uint32_t kF64InfoOff = kF64HdrOff + sizeof(StageHdr);
constexpr uint32_t kF64NextOff = kF64InfoOff + sizeof(TileInfo);
constexpr uint32_t kF64BatchStageBytes = (kF64NextOff + sizeof(ETileSrc) + 127) / 128 * 128;
constexpr size_t kF64BatchStageSmem = 2 * static_cast<size_t>(kF64BatchStageBytes) + 16;
static_assert(sizeof(InstanceDesc) % 16 == 0, "16-byte copies");

// double row r (as f64_stage_row) of a batch tile in global memory
__device__ __forceinline__ const double* f64_tile_row(const ETileSrc& src, int r) {
    const int64_t ep = src.ne_pad;
    if (r < 6) return static_cast<const double*>(src.sigma) + r * ep;
    if (r < 18) return static_cast<const double*>(src.qia) + (r - 6) * ep;
    if (r == 18) return static_cast<const double*>(src.vol0);
    if (r == 19) return static_cast<const double*>(src.cbrt_v0);
    if (r == 20) return static_cast<const double*>(src.cbrt_v0sq);
    if (r == 21) return static_cast<const double*>(src.eps_p);
    return static_cast<const double*>(src.bt) + (r - kF64StageRows) * ep;
}

__device__ __forceinline__ void f64_batch_stage_issue(const BatchTables& T, const ETileSrc& src, int64_t t_next,
                                                      int64_t ntiles, unsigned char* stage, uint32_t dst, uint32_t bar,
                                                      int lane) {
    constexpr int drows = kF64StageRows + 24;
    const uint32_t cnt = static_cast<uint32_t>(src.cnt);
    const bool next = t_next < ntiles;
    if (lane == 0) {
        TileInfo* ti = reinterpret_cast<TileInfo*>(stage + kF64InfoOff);
        ti->slot = src.slot;
        ti->base = src.base;
        mbar_arrive_expect_tx(bar, f64_stage_tx_bytes<true, true>(cnt) + sizeof(InstanceDesc) + sizeof(StageHdr) +
                                       (next ? sizeof(ETileSrc) : 0u));
    }
    __syncwarp();
    fence_proxy_async_smem();  // the block's reads of this stage come before the copies into it
    const uint32_t dbase = dst + 8u * kF64BatchTile * 4u;
    for (int q = lane; q < 8 + drows + 3; q += 32) {
        if (q < 8)
            bulk_g2s(dst + q * (kF64BatchTile * 4u), static_cast<const uint32_t*>(src.conn) + q * src.ne_pad,
                     cnt * 4u, bar);
        else if (q < 8 + drows)
            bulk_g2s(dbase + (q - 8) * (kF64BatchTile * 8u), f64_tile_row(src, q - 8), cnt * 8u, bar);
        else if (q == 8 + drows)
            bulk_g2s(dst + kF64DescOff, T.desc + src.slot, sizeof(InstanceDesc), bar);
        else if (q == 8 + drows + 1)
            bulk_g2s(dst + kF64HdrOff, T.sparam + src.slot, sizeof(StageHdr), bar);
        else if (next)
            bulk_g2s(dst + kF64NextOff, T.etile_src + t_next, sizeof(ETileSrc), bar);
    }
}

// The batched FP64 element pass: element_body's arithmetic per element, so
// states are bit-identical to the single-instance pass.  A block's
// consecutive tiles of one instance form a run whose sums and minima are
// reduced once, into the partial slot of the run's first tile.
__global__ void __launch_bounds__(kF64BatchTile, 256 / kF64BatchTile) k_element_batch_fp64(BatchTables T) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int TT = kF64BatchTile;
    constexpr int NW = TT / 32;
    constexpr uint32_t SB = kF64BatchStageBytes;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t stage0 = smem_addr(smem);
    const uint32_t bar0 = stage0 + 2 * SB;
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
                f64_batch_stage_issue(T, src, t + 2 * gstride, ntiles, smem + s * SB, stage0 + s * SB, bar0 + 8 * s,
                                      lane);
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
        unsigned char* st = smem + s * SB;
        const InstanceDesc& d = *reinterpret_cast<const InstanceDesc*>(st + kF64DescOff);
        const StageHdr& h = *reinterpret_cast<const StageHdr*>(st + kF64HdrOff);
        const TileInfo& ti = *reinterpret_cast<const TileInfo*>(st + kF64InfoOff);
        if (ti.slot != run_slot) {
            flush();
            run_slot = ti.slot;
            run_tile = t;
            run_ctl = d.ctl;
            run_live = h.live != 0;
        }
        const int64_t e = static_cast<int64_t>(ti.base) + tid;
        if (run_live && e < d.E.ne) {
            // arrays copied to registers, material read at use
            const ElemArrays E = d.E;
            const NodeArrays N = d.N;
            const double dt1 = h.dt1;
            const double* dr = reinterpret_cast<const double*>(st + 8 * TT * 4);
            const Fp64Src S{reinterpret_cast<const uint32_t*>(st), dr, dr + 6 * TT, dr + 18 * TT, dr + 19 * TT,
                            dr + 20 * TT, dr + 21 * TT, TT, tid, dr + kF64StageRows * TT, TT, tid};
            double d1, l1;
            element_body<true, false, true, true, ENSC_F64_PREFETCH>(E, N, d.M, S, dt1, e, d1, l1, ei, eh, ev, bad);
            dts = d1 < dts ? d1 : dts;
            len = l1 < len ? l1 : len;
        }
        __syncthreads();  // the block is done with stage s
        const int64_t tn = t + 2 * gstride;
        if (wid == 0 && tn < ntiles) {
            const ETileSrc src = *reinterpret_cast<const ETileSrc*>(st + kF64NextOff);
            f64_batch_stage_issue(T, src, tn + 2 * gstride, ntiles, st, stage0 + s * SB, bar, lane);
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

// As k_node_batch_mixed: one warp per node tile, slots and first nodes read
// two tiles ahead, table lines prefetched into L1 one tile ahead.
template <int NT>
__global__ void __launch_bounds__(NT, ENSC_NODE_MINB_FP64 * kNodeThreads / NT) k_node_batch_fp64(BatchTables T) {
    constexpr int W = kNodeGroupFp64;
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
                if (v.grouped) {
                    node_group<W>(v, dt_i, dt_i_1, amp, n0, kin, wext, bad);
                } else {
                    const InstanceDesc& d = T.desc[slot];
                    for (int j = 0; j < W && n0 + j < v.nn; ++j)
                        node_body(d.E, d.N, d.M, dt_i, dt_i_1, amp, n0 + j, kin, wext, bad);
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

namespace {
constexpr bool kStagedBt = ENSC_STAGED_FP64 == 2;
}

void launch_element_fp64(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl, const Partials& P,
                         int grid, bool init, cudaStream_t st) {
    if (ENSC_WARP_PIPE_FP64 && !init && E.tiles_aligned) {
        if (M.plastic) k_element_fp64_warp<true><<<grid, 32 * kF64PipeWarps, kF64WarpPipeSmem, st>>>(E, N, M, ctl, P);
        else k_element_fp64_warp<false><<<grid, 32 * kF64PipeWarps, kF64WarpPipeSmem, st>>>(E, N, M, ctl, P);
        return;
    }
    if (ENSC_STAGED_FP64 && !init && E.tiles_aligned) {
        constexpr size_t smem = f64_stage_smem<kStagedBt>();
        if (M.plastic) k_element_staged<true, kStagedBt><<<grid, kStageTileF64, smem, st>>>(E, N, M, ctl, P);
        else k_element_staged<false, kStagedBt><<<grid, kStageTileF64, smem, st>>>(E, N, M, ctl, P);
        return;
    }
    if (M.plastic) {
        if (init) k_element<true, true><<<grid, kElemThreads, 0, st>>>(E, N, M, ctl, P);
        else k_element<true, false><<<grid, kElemThreads, 0, st>>>(E, N, M, ctl, P);
    } else {
        if (init) k_element<false, true><<<grid, kElemThreads, 0, st>>>(E, N, M, ctl, P);
        else k_element<false, false><<<grid, kElemThreads, 0, st>>>(E, N, M, ctl, P);
    }
}

void launch_node_fp64(const ElemArrays& E, const NodeArrays& N, const Material& M, Ctl* ctl, const Partials& P,
                      int grid, cudaStream_t st) {
    k_node<<<grid, kNodeThreads, 0, st>>>(E, N, M, ctl, P);
}

int occupancy_element_fp64(bool plastic) {
    int nb = 0;
    if (ENSC_WARP_PIPE_FP64) {
        cudaFuncSetAttribute(k_element_fp64_warp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kF64WarpPipeSmem));
        cudaFuncSetAttribute(k_element_fp64_warp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kF64WarpPipeSmem));
        if (plastic)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_fp64_warp<true>, 32 * kF64PipeWarps,
                                                          kF64WarpPipeSmem);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_fp64_warp<false>, 32 * kF64PipeWarps,
                                                          kF64WarpPipeSmem);
        return nb;
    }
    if (ENSC_STAGED_FP64) {
        // more than the default 48 KB of dynamic shared memory: set on the
        // current device, before any launch or capture
        constexpr size_t smem = f64_stage_smem<kStagedBt>();
        cudaFuncSetAttribute(k_element_staged<true, kStagedBt>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        cudaFuncSetAttribute(k_element_staged<false, kStagedBt>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        if (plastic)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_staged<true, kStagedBt>, kStageTileF64, smem);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_staged<false, kStagedBt>, kStageTileF64, smem);
        return nb;
    }
    if (plastic) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element<true, false>, kElemThreads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element<false, false>, kElemThreads, 0);
    return nb;
}

void launch_acceleration_fp64(const ElemArrays& E, const NodeArrays& N, const Material& M, const Ctl* ctl,
                              double* a_aos, cudaStream_t st) {
    const int64_t g = std::min<int64_t>((N.nn + kNodeThreads - 1) / kNodeThreads, 65535);
    k_acceleration<<<static_cast<int>(g), kNodeThreads, 0, st>>>(E, N, M, ctl, a_aos);
}

int node_group_width(bool mixed_precision) { return mixed_precision ? kNodeGroupMixed : kNodeGroupFp64; }

int occupancy_node_fp64() {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_node, kNodeThreads, 0);
    return nb;
}


void launch_element_batch_fp64(const BatchTables& T, int grid, cudaStream_t st) {
    k_element_batch_fp64<<<grid, kF64BatchTile, kF64BatchStageSmem, st>>>(T);
}
void launch_node_batch_fp64(const BatchTables& T, int grid, int threads, cudaStream_t st) {
    if (threads == kNodeThreads / 2) k_node_batch_fp64<kNodeThreads / 2><<<grid, threads, 0, st>>>(T);
    else k_node_batch_fp64<kNodeThreads><<<grid, kNodeThreads, 0, st>>>(T);
}
int occupancy_element_batch_fp64() {
    int nb = 0;
    // dynamic shared memory above the default 48 KB: set on the current
    // device before any launch or capture
    cudaFuncSetAttribute(k_element_batch_fp64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(kF64BatchStageSmem));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_element_batch_fp64, kF64BatchTile, kF64BatchStageSmem);
    return nb;
}

int batch_element_tile_fp64() { return kF64BatchTile; }
int occupancy_node_batch_fp64(int threads) {
    int nb = 0;
    if (threads == kNodeThreads / 2)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_node_batch_fp64<kNodeThreads / 2>, threads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_node_batch_fp64<kNodeThreads>, kNodeThreads, 0);
    return nb;
}

}  // namespace ensc
