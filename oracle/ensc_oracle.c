/* Test infrastructure -- NOT part of the product.  See ensc_oracle.h.
 *
 * Plain-C restatement of the EnSCDynamics explicit stepper.  Every routine
 * cites the reference function it follows (paths relative to the reference
 * project).  Floating-point evaluation order is fixed and documented here;
 * the product's FP64 CUDA kernel evaluates the same expressions in the same
 * order (explicit fused multiply-adds only, no contraction), so the two
 * agree bit-for-bit:
 *   - sums over the 8 element nodes run node by node with fma; the 3- and
 *     4-term dot products are spelled out with fma at each site;
 *   - 3x3 determinant and inverse follow Eigen 3.4's closed forms
 *     (Eigen/src/LU/Determinant.h bruteforce_det3_helper and
 *     Eigen/src/LU/InverseImpl.h compute_inverse<...,3>), the library the
 *     reference links.
 * Compiled with -ffp-contract=off so only the explicit fma() calls fuse.
 */
#include "ensc_oracle.h"

#include <float.h>
#include <math.h>
#include <string.h>

/* Hourglass base vectors Gamma (exDyna3D.cpp:1003-1008), rows k=0..3. */
static const double TAU[4][8] = {
    {1., -1., 1., -1., 1., -1., 1., -1.},
    {-1., -1., 1., 1., 1., 1., -1., -1.},
    {-1., 1., 1., -1., 1., -1., -1., 1.},
    {-1., 1., -1., 1., 1., -1., 1., -1.},
};

/* Reference-element node coordinates (Element_HexN8.cpp:49-91). */
static const double XI[8][3] = {
    {-1., -1., -1.}, {1., -1., -1.}, {1., 1., -1.}, {-1., 1., -1.},
    {-1., -1., 1.},  {1., -1., 1.},  {1., 1., 1.},  {-1., 1., 1.},
};

void ensc_oracle_material_update(ensc_oracle_params* p) {
    /* Material_elastic::update (Material_elastic.cpp:9-14) */
    p->G = p->E / ((1.0 + p->nu) * 2.0);
    p->K = p->E / (1.0 - 2.0 * p->nu) / 3.0;
    p->lambda = 2.0 * p->G * p->nu / (1.0 - 2.0 * p->nu);
    p->wos = sqrt((p->lambda + 2.0 * p->G) / p->rho);
}

/* Eigen 3.4 bruteforce 3x3 determinant: h(0,1,2) - h(1,0,2) + h(2,0,1),
 * h(a,b,c) = m(0,a) * (m(1,b)*m(2,c) - m(1,c)*m(2,b)). */
double ensc_oracle_amplitude(const double* amp, int32_t n, double time, double dt) {
    /* Restated from deal_amp with its behaviour kept as is: the scan stops at
     * the first segment whose end lies before `time` (the factor is then 1),
     * a cycle inside one segment takes the segment's value at mid-cycle,
     * and a cycle that crosses segment ends takes the mean of the piecewise
     * linear curve over [time, time + dt], where the partial last segment
     * uses the first segment's slope in its intercept (exDyna3D.cpp:1257)
     * and time beyond the last point counts with value 1 (:1266-1270).
     * n < 2: factor 1. */
    double y = 1.0;
    for (int32_t i = 0; i + 1 < n; ++i) {
        const double x1 = amp[2 * i], y1 = amp[2 * i + 1];
        const double x2 = amp[2 * i + 2], y2 = amp[2 * i + 3];
        if (time > x2) break;
        const double m = (y2 - y1) / (x2 - x1);
        const double c = y1 - m * x1;
        const double x = time + dt / 2.0;
        if ((x + dt / 2.0) < x2) {
            y = m * x + c;
            break;
        }
        const double dt1 = x2 - time;
        const double xm = time + dt1 / 2.0;
        const double ym = m * xm + c;
        const double a1 = ym * dt1;
        double a2 = 0.0;
        for (int32_t j = 2; j + i < n; ++j) {
            const double xj = amp[2 * (i + j)], yj = amp[2 * (i + j) + 1];
            const double xp = amp[2 * (i + j - 1)], yp = amp[2 * (i + j - 1) + 1];
            if ((x + dt / 2.0) > xj) {
                a2 += (xj - xp) * (yj + yp) / 2.0;
            } else {
                const double mj = (yj - yp) / (xj - xp);
                const double cj = yp - m * xp;
                const double yend = mj * (x + dt / 2.0) + cj;
                a2 += (x + dt / 2.0 - xp) * (yp + yend) / 2.0;
                break;
            }
        }
        const double x_end = amp[2 * (n - 1)];
        if (x + dt / 2.0 > x_end) a2 += (x + dt / 2.0 - x_end) * 1.0;
        y = (a1 + a2) / dt;
        break;
    }
    return y;
}

static double det3(const double m[3][3]) {
    const double h0 = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]);
    const double h1 = m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    const double h2 = m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    return (h0 - h1) + h2;
}

static double cof3(const double m[3][3], int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m[i1][j1] * m[i2][j2] - m[i1][j2] * m[i2][j1];
}

/* Eigen 3.4 compute_inverse<...,3>: det from cofactor column 0 summed left to
 * right, inv(i,j) = cofactor(j,i) * (1/det). */
static void inv3(const double m[3][3], double r[3][3]) {
    const double c0 = cof3(m, 0, 0), c1 = cof3(m, 1, 0), c2 = cof3(m, 2, 0);
    const double det = (c0 * m[0][0] + c1 * m[1][0]) + c2 * m[2][0];
    const double invdet = 1.0 / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r[i][j] = cof3(m, j, i) * invdet;
}

void ensc_oracle_setup(int64_t nn, int64_t ne, const uint32_t* conn, const double* x0, double rho,
                       double* bt, double* vol0, double* cbrt_v0, double* cbrt_v0sq,
                       double* inv_mass) {
    /* dN/dxi at the single Gauss point xi = 0 (fevalues.h:201-212,
     * Element_HexN8.cpp:156-164): (1/8) * xi_i * (1 + 0) * (1 + 0). */
    double dn[3][8];
    for (int a = 0; a < 8; ++a)
        for (int d = 0; d < 3; ++d) dn[d][a] = 1.0 / 8.0 * XI[a][d];
    for (int64_t i = 0; i < 3 * nn; ++i) inv_mass[i] = 0.0;
    for (int64_t e = 0; e < ne; ++e) {
        double xyz[8][3];
        for (int a = 0; a < 8; ++a)
            for (int c = 0; c < 3; ++c) xyz[a][c] = x0[3 * (int64_t)conn[8 * e + a] + c];
        /* jacobi = dN * xyz (fevalues.h:252) */
        double jac[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double s = dn[r][0] * xyz[0][c];
                for (int k = 1; k < 8; ++k) s += dn[r][k] * xyz[k][c];
                jac[r][c] = s;
            }
        double ij[3][3];
        inv3(jac, ij);
        const double detj = det3(jac);
        /* B = J^-1 dN (fevalues.h:260-263); all_BT = B^T (exDyna3D.cpp:504) */
        for (int a = 0; a < 8; ++a)
            for (int r = 0; r < 3; ++r)
                bt[24 * e + 3 * a + r] = (ij[r][0] * dn[0][a] + ij[r][1] * dn[1][a]) + ij[r][2] * dn[2][a];
        /* JxW with the 1-point weight 2*2*2 (gauss_integral_1d.cpp:37-39) */
        const double v0 = detj * 8.0;
        vol0[e] = v0;
        cbrt_v0[e] = cbrt(v0);
        cbrt_v0sq[e] = cbrt(v0 * v0);
        const double node_mass = rho * v0 / 8.0;
        for (int a = 0; a < 8; ++a)
            for (int c = 0; c < 3; ++c) inv_mass[3 * (int64_t)conn[8 * e + a] + c] += node_mass;
    }
    for (int64_t i = 0; i < 3 * nn; ++i) inv_mass[i] = 1.0 / inv_mass[i];
}

void ensc_oracle_cbrt_pair(int64_t ne, const double* vol0, double* cbrt_v0, double* cbrt_v0sq) {
    for (int64_t e = 0; e < ne; ++e) {
        cbrt_v0[e] = cbrt(vol0[e]);
        cbrt_v0sq[e] = cbrt(vol0[e] * vol0[e]);
    }
}

/* min_ele_edge (exDyna3D.cpp:1173-1220): 12 edges, squared lengths compared in
 * the order bottom ring, top ring, verticals; sqrt of the minimum. */
static double min_edge(const double xyz[8][3]) {
    double m = DBL_MAX;
    static const int E0[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
    static const int E1[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
    for (int k = 0; k < 12; ++k) {
        const double dx = xyz[E1[k]][0] - xyz[E0[k]][0];
        const double dy = xyz[E1[k]][1] - xyz[E0[k]][1];
        const double dz = xyz[E1[k]][2] - xyz[E0[k]][2];
        const double t = fma(dz, dz, fma(dy, dy, dx * dx));
        if (t < m) m = t;
    }
    return sqrt(m);
}

static void gather_xyz(const ensc_oracle_state* s, int64_t e, double xyz[8][3]) {
    for (int a = 0; a < 8; ++a)
        for (int c = 0; c < 3; ++c) xyz[a][c] = s->x[3 * (int64_t)s->conn[8 * e + a] + c];
}

/* One element of add_inForce_to_rhs (exDyna3D.cpp:556-573): kinematics
 * (reinit_some_CellData :888-918), Jaumann stress (:920-998) with the optional
 * J2 return, hourglass (:1000-1071), bulk viscosity (:1073-1109) and the
 * element dt (:828-834).  Writes the 8x3 element force f; returns dtStable.
 * de[0..2] receive the element's internal/hourglass/viscous work increments.
 *
 * The same quantities as the reference, regrouped so the per-node work is
 * a few accumulations (shared with the GPU kernel, operation for operation):
 *   L0  = v_e B0^T                 (3x3, sum over nodes)
 *   VT  = v_e Gamma^T              (3x4, signed sums, exact)
 *   L   = L0 F^-1                  (= v_e b^T, :928)
 *   HIA = VT - L0 TX^T             (= v_e ATAU^T with ATAU = Gamma - TX B0, :1020-1021)
 *   Gq  = QIA + CR HIA             (hourglass force h_j = ATAU_j^T Gq, :1053-1067)
 *   W   = Gq TX                    (3x3)
 *   Z   = Vc F^-1 (sigma - p I) - W^T
 *   f_j = -(B0_j Z) - Gamma_j Gq^T (= -b_j sigma V - h_j + p b_j V, :985-997, :1070, :1106)
 * Sums over the 8 nodes run node by node from 0.0 with fma (one rounding per
 * term); short dot products are spelled out with fma at each site. */
static double element(const ensc_oracle_params* p, ensc_oracle_state* s, int64_t e, double dt1,
                      double f[8][3], double de[3]) {
    const uint32_t* cn = s->conn + 8 * e;
    const double* BT = s->bt + 24 * e; /* BT[3*a + c] */
    double vel[3][8], xyz[8][3], ue[3][8];
    for (int a = 0; a < 8; ++a) {
        const int64_t n = cn[a];
        for (int c = 0; c < 3; ++c) {
            vel[c][a] = s->v[3 * n + c];
            xyz[a][c] = s->x[3 * n + c];
            ue[c][a] = s->u[3 * n + c];
        }
    }
    /* hourglass base projections TX = Gamma xyz (exact: entries are +-1) */
    double TX[4][3];
    for (int k = 0; k < 4; ++k)
        for (int c = 0; c < 3; ++c) {
            double t = TAU[k][0] > 0 ? xyz[0][c] : -xyz[0][c];
            for (int j = 1; j < 8; ++j) t = TAU[k][j] > 0 ? t + xyz[j][c] : t - xyz[j][c];
            TX[k][c] = t;
        }
    /* F = I + u_e B0^T (:862-865) */
    double F[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double t = 0.0;
            for (int k = 0; k < 8; ++k) t = fma(ue[r][k], BT[3 * k + c], t);
            F[r][c] = (r == c) ? 1.0 + t : t;
        }
    const double J = det3(F); /* :867-870 */
    double Fi[3][3];
    inv3(F, Fi);
    /* per-node accumulations */
    double L0[3][3] = {{0.0}}, VT[3][4] = {{0.0}}, nx2 = 0.0;
    for (int j = 0; j < 8; ++j) {
        const double b0 = BT[3 * j], b1 = BT[3 * j + 1], b2 = BT[3 * j + 2];
        const double bb[3] = {b0, b1, b2};
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) L0[r][c] = fma(vel[r][j], bb[c], L0[r][c]);
            for (int k = 0; k < 4; ++k) VT[r][k] = TAU[k][j] > 0 ? VT[r][k] + vel[r][j] : VT[r][k] - vel[r][j];
        }
        nx2 = nx2 + fma(b2, b2, fma(b1, b1, b0 * b0));
    }
    double L[3][3], HIA[3][4];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) L[r][c] = fma(L0[r][2], Fi[2][c], fma(L0[r][1], Fi[1][c], L0[r][0] * Fi[0][c]));
        for (int k = 0; k < 4; ++k)
            HIA[r][k] = VT[r][k] - fma(L0[r][2], TX[k][2], fma(L0[r][1], TX[k][1], L0[r][0] * TX[k][0]));
    }
    /* VolRate = tr L (:877-885) */
    const double vr = (L[0][0] + L[1][1]) + L[2][2];
    double eps[6];
    eps[0] = L[0][0];
    eps[1] = L[1][1];
    eps[2] = L[2][2];
    eps[3] = (L[0][1] + L[1][0]) / 2.0;
    eps[4] = (L[0][2] + L[2][0]) / 2.0;
    eps[5] = (L[1][2] + L[2][1]) / 2.0;
    for (int i = 0; i < 6; ++i) eps[i] *= dt1;
    const double w0 = (L[0][1] - L[1][0]) / 2.0;
    const double w1 = (L[0][2] - L[2][0]) / 2.0;
    const double w2 = (L[1][2] - L[2][1]) / 2.0;
    const double lam = p->lambda, G = p->G;
    const double tr = (eps[0] + eps[1]) + eps[2];
    double jau[6];
    jau[0] = lam * tr + 2.0 * G * eps[0];
    jau[1] = lam * tr + 2.0 * G * eps[1];
    jau[2] = lam * tr + 2.0 * G * eps[2];
    jau[3] = 2.0 * G * eps[3];
    jau[4] = 2.0 * G * eps[4];
    jau[5] = 2.0 * G * eps[5];
    double* sg = s->sigma + 6 * e;
    double inc[6];
    inc[0] = jau[0] + 2.0 * sg[3] * w0 * dt1 + 2.0 * sg[4] * w1 * dt1;
    inc[1] = jau[1] - 2.0 * sg[3] * w0 * dt1 + 2.0 * sg[5] * w2 * dt1;
    inc[2] = jau[2] - 2.0 * sg[4] * w1 * dt1 - 2.0 * sg[5] * w2 * dt1;
    inc[3] = jau[3] + (sg[1] - sg[0]) * w0 * dt1 + sg[5] * w1 * dt1;
    inc[4] = jau[4] + (sg[2] - sg[0]) * w1 * dt1 + sg[5] * w0 * dt1;
    inc[5] = jau[5] + (sg[2] - sg[1]) * w2 * dt1 + sg[3] * w1 * dt1 - sg[4] * w0 * dt1;
    double sold[6];
    for (int i = 0; i < 6; ++i) {
        sold[i] = sg[i];
        sg[i] += inc[i];
    }
    /* J2 radial return with linear isotropic hardening (no reference
     * counterpart; skipped entirely when yield0 <= 0, so the elastic path is
     * the reference's own update). */
    if (p->yield0 > 0.0) {
        const double pm = ((sg[0] + sg[1]) + sg[2]) / 3.0;
        const double d0 = sg[0] - pm, d1 = sg[1] - pm, d2 = sg[2] - pm;
        const double j2 = 0.5 * ((d0 * d0 + d1 * d1) + d2 * d2) + ((sg[3] * sg[3] + sg[4] * sg[4]) + sg[5] * sg[5]);
        const double seq = sqrt(3.0 * j2);
        const double sy = p->yield0 + p->hardening * s->eps_p[e];
        if (seq > sy) {
            const double dl = (seq - sy) / (3.0 * G + p->hardening);
            const double r = 1.0 - 3.0 * G * dl / seq;
            sg[0] = d0 * r + pm;
            sg[1] = d1 * r + pm;
            sg[2] = d2 * r + pm;
            sg[3] *= r;
            sg[4] *= r;
            sg[5] *= r;
            s->eps_p[e] += dl;
        }
    }
    const double V0 = s->vol0[e];
    const double Vc = J * V0;
    /* stress work: V * (sigma_mid : d_eps), shear terms doubled */
    {
        double w = 0.0;
        for (int i = 0; i < 6; ++i) {
            const double sm = 0.5 * (sold[i] + sg[i]);
            w += (i < 3 ? 1.0 : 2.0) * sm * eps[i];
        }
        de[0] = w * Vc;
    }
    /* hourglass coefficients and history (:1038-1050) */
    const double C2 = 0.1;
    const double r43 = 4.0 / 3.0;
    const double r1s8 = 1.0 / sqrt(8.0);
    const double DR = p->c_dr * (r43 * G + p->K) * C2 * nx2 * Vc * r1s8 * dt1;
    const double CR = p->c_cr * p->rho * V0 / Vc * s->cbrt_v0sq[e] * p->wos / 4.0;
    double* Q = s->qia + 12 * e;
    double Gq[3][4];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 4; ++k) {
            Q[4 * i + k] = fma(DR, HIA[i][k], Q[4 * i + k]);
            Gq[i][k] = fma(CR, HIA[i][k], Q[4 * i + k]);
        }
    /* bulk viscosity pressure (:1073-1109) */
    const int visc = !(fabs(vr) < 1.0e-10);
    double pv = 0.0;
    de[2] = 0.0;
    if (visc) {
        const double rho_c = p->rho / J;
        const double len0 = s->cbrt_v0[e];
        const double m0 = vr < 0.0 ? vr : 0.0; /* std::min(zero, VolRate) */
        pv = rho_c * len0 * (p->cvisq * p->cvisq * len0 * vr * m0 - p->cvisl * p->wos * vr);
        de[2] = -(pv * Vc * vr) * dt1;
    }
    /* Z = Vc F^-1 (sigma - p I) - W^T,  W = Gq TX */
    const double Sp[3][3] = {{sg[0] - pv, sg[3], sg[4]}, {sg[3], sg[1] - pv, sg[5]}, {sg[4], sg[5], sg[2] - pv}};
    double Z[3][3], W[3][3];
    for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c)
            W[i][c] = fma(Gq[i][3], TX[3][c], fma(Gq[i][2], TX[2][c], fma(Gq[i][1], TX[1][c], Gq[i][0] * TX[0][c])));
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 3; ++i)
            Z[c][i] = Vc * fma(Fi[c][2], Sp[2][i], fma(Fi[c][1], Sp[1][i], Fi[c][0] * Sp[0][i])) - W[i][c];
    /* nodal forces f_j = -(B0_j Z) - Gamma_j Gq^T */
    for (int j = 0; j < 8; ++j) {
        const double b0 = BT[3 * j], b1 = BT[3 * j + 1], b2 = BT[3 * j + 2];
        for (int i = 0; i < 3; ++i) {
            double tg = TAU[0][j] > 0 ? Gq[i][0] : -Gq[i][0];
            for (int k = 1; k < 4; ++k) tg = TAU[k][j] > 0 ? tg + Gq[i][k] : tg - Gq[i][k];
            f[j][i] = -fma(b2, Z[2][i], fma(b1, Z[1][i], b0 * Z[0][i])) - tg;
        }
    }
    /* hourglass power sum_j h_j . v_j = Gq : HIA */
    {
        double hp = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 4; ++k) hp = fma(Gq[i][k], HIA[i][k], hp);
        de[1] = hp * dt1;
    }
    /* compute_dtStable (:828-834) with this cycle's min edge */
    {
        const double Len = s->len[e];
        const double cd = p->wos;
        const double m0 = vr < 0.0 ? vr : 0.0;
        const double xi = p->cvisl - p->cvisq * p->cvisq * Len / cd * m0;
        return (sqrt(1.0 + xi * xi) - xi) * Len / cd;
    }
}

/* add_inForce_to_rhs (exDyna3D.cpp:517-640): element loop scattering each
 * element's 8 nodal forces into 8 per-local-slot vectors, then the fixed-order
 * sum ((((((a0+a1)+a2)+a3)+a4)+a5)+a6)+a7. */
static void force_pass(const ensc_oracle_params* p, ensc_oracle_state* s, double dt1, double de_sum[3]) {
    const int64_t ndof = 3 * s->nn;
    memset(s->slots, 0, sizeof(double) * 8 * (size_t)ndof);
    de_sum[0] = de_sum[1] = de_sum[2] = 0.0;
    for (int64_t e = 0; e < s->ne; ++e) {
        double f[8][3], de[3];
        s->dtstable[e] = element(p, s, e, dt1, f, de);
        for (int a = 0; a < 8; ++a)
            for (int c = 0; c < 3; ++c) s->slots[a * ndof + 3 * (int64_t)s->conn[8 * e + a] + c] += f[a][c];
        de_sum[0] += de[0];
        de_sum[1] += de[1];
        de_sum[2] += de[2];
    }
    for (int64_t i = 0; i < ndof; ++i) {
        double t = s->slots[i];
        for (int a = 1; a < 8; ++a) t += s->slots[a * ndof + i];
        s->force[i] = t;
    }
}

static void update_lengths(ensc_oracle_state* s, double* minlen) {
    double m = DBL_MAX;
    for (int64_t e = 0; e < s->ne; ++e) {
        double xyz[8][3];
        gather_xyz(s, e, xyz);
        s->len[e] = min_edge(xyz);
        if (s->len[e] < m) m = s->len[e];
    }
    *minlen = m;
}

void ensc_oracle_init_pass(const ensc_oracle_params* p, ensc_oracle_state* s) {
    double ml, de[3];
    update_lengths(s, &ml);
    force_pass(p, s, 0.0, de);
}

void ensc_oracle_apply_bc_v(ensc_oracle_state* s) {
    /* velocity BCs first, then fixed DOFs (exDyna3D.cpp:386-487) */
    const int64_t ndof = 3 * s->nn;
    for (int64_t i = 0; i < ndof; ++i)
        if (s->bc_code[i] & 2) s->v[i] = s->bc_value[i];
    for (int64_t i = 0; i < ndof; ++i)
        if (s->bc_code[i] & 1) s->v[i] = 0.0;
}

double ensc_oracle_kinetic(const ensc_oracle_state* s) {
    double k = 0.0;
    for (int64_t i = 0; i < 3 * s->nn; ++i) k += 0.5 * (s->v[i] * s->v[i]) / s->inv_mass[i];
    return k;
}

int64_t ensc_oracle_cycles(const ensc_oracle_params* p, ensc_oracle_state* s, int64_t max_cycles,
                           double step_end) {
    const int64_t ndof = 3 * s->nn;
    int64_t done = 0;
    while (s->time < step_end && done < max_cycles) {
        /* update_minVertex_perMaterial_and_dt (exDyna3D.cpp:663-686) */
        double minlen;
        update_lengths(s, &minlen);
        s->dt_i_1 = s->dt_i;
        const double time_prev = s->time + s->dt_i_1;
        double dt = minlen / p->wos;
        double tmp = DBL_MAX;
        for (int64_t e = 0; e < s->ne; ++e)
            if (s->dtstable[e] < tmp) tmp = s->dtstable[e];
        dt = dt < tmp ? dt : tmp;
        dt *= p->factor;
        s->dt_i = dt;
        if ((p->total_time - time_prev) < s->dt_i && (p->total_time - time_prev) > 0.0) {
            s->dt_i = p->total_time - time_prev;
            s->dt_i_1 = s->dt_i;
        }
        /* last-step clamp of run() (exDyna3D.cpp:90-97) */
        if (s->time + s->dt_i_1 > step_end) {
            const double rem = step_end - s->time;
            s->dt_i = s->dt_i_1 = rem;
        }
        /* computeSate (exDyna3D.cpp:774-793) */
        s->time += s->dt_i_1;
        if (s->time > p->total_time) s->time = p->total_time;
        ensc_oracle_apply_bc_v(s);
        double de[3];
        force_pass(p, s, s->dt_i_1, de);
        s->energy[1] += de[0];
        s->energy[2] += de[1];
        s->energy[3] += de[2];
        const double dt_avg = (s->dt_i + s->dt_i_1) / 2.0;
        double wext = 0.0, kin = 0.0;
        const double ampv = (p->gravity_on && p->amp_n > 0) ? ensc_oracle_amplitude(p->amp, p->amp_n, s->time, s->dt_i)
                                                            : 1.0;
        for (int64_t i = 0; i < ndof; ++i) {
            double a = s->force[i];
            double g = 0.0;
            if (p->gravity_on) { /* apply_gravity (:809-824) */
                g = ampv * p->gravity_value * p->gravity_dir[i % 3] / s->inv_mass[i];
                a += g;
            }
            /* apply_boundary_condition_a (:2029-2145) */
            s->rf[i] = 0.0;
            const int8_t code = s->bc_code[i];
            double r = 0.0;
            if (code & 2) {
                r = -a;
                a = 0.0;
            }
            if ((code & 1) && a != 0.0) {
                s->rf[i] = -a;
                r = -a;
                a = 0.0;
            }
            /* compute_a, update_velocity, update_displacement, move_mesh
             * (:642-654, :688-696) */
            a = a * s->inv_mass[i];
            const double vold = s->v[i];
            s->v[i] += (s->dt_i + s->dt_i_1) * a / 2.0;
            s->u[i] += s->dt_i * s->v[i];
            s->x[i] += s->dt_i * s->v[i];
            const double vbar = 0.5 * (vold + s->v[i]);
            wext += (g + r) * dt_avg * vbar;
            kin += 0.5 * (s->v[i] * s->v[i]) / s->inv_mass[i];
        }
        s->energy[4] += wext;
        s->energy[0] = kin;
        ++s->cycles;
        ++done;
    }
    return done;
}
