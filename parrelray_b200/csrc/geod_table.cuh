// geod_table.cuh - geodesic acceleration from the full Christoffel table of
// the Kerr-Schild metric, the way a metric plug-in author writes it
// (d_k g_mn -> Gamma_{lmn} -> g^{kl} Gamma_{lmn} -> contraction).  Used by the
// PLAIN schedule (the reference's structure) and for A/B comparisons with
// the register-resident contraction geod_ks().
#pragma once
#include "prr_device.cuh"

namespace prr {

template <class T> __device__ __noinline__ V4<T> geod_table(const V4<T> &p, const V4<T> &u, T M, T a)
{
    if (M == (T)0) return {0, 0, 0, 0};
    T x = p.x, y = p.y, z = p.z;
    T R2 = x * x + y * y + z * z, a2 = a * a, b = R2 - a2;
    T S = sqrt(b * b + (T)4 * a2 * z * z);
    T r2 = (T)0.5 * (b + S), r = sqrt(r2);
    T dr[3] = {x * r / S, y * r / S, z * (r2 + a2) / (r * S)};
    T q = r2 + a2, Sig = r2 * r2 + a2 * z * z;
    T f = (T)2 * M * r2 * r / Sig;
    T df[3], l[4], dl[4][3];
    for (int k = 0; k < 3; k++) {
        T dSig = (T)4 * r2 * r * dr[k] + (k == 2 ? (T)2 * a2 * z : (T)0);
        df[k] = (T)2 * M * ((T)3 * r2 * dr[k] * Sig - r2 * r * dSig) / (Sig * Sig);
    }
    T nx = r * x + a * y, ny = r * y - a * x;
    l[0] = nx / q; l[1] = ny / q; l[2] = z / r; l[3] = 1;
    for (int k = 0; k < 3; k++) {
        T dq = (T)2 * r * dr[k];
        T dnx = dr[k] * x + (k == 0 ? r : (T)0) + (k == 1 ? a : (T)0);
        T dny = dr[k] * y + (k == 1 ? r : (T)0) - (k == 0 ? a : (T)0);
        dl[0][k] = (dnx * q - nx * dq) / (q * q);
        dl[1][k] = (dny * q - ny * dq) / (q * q);
        dl[2][k] = (k == 2 ? (T)1 / r : (T)0) - z * dr[k] / r2;
        dl[3][k] = 0;
    }
    T dg[4][4][4];
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) {
            for (int k = 0; k < 3; k++) dg[m][n][k] = df[k] * l[m] * l[n] + f * (dl[m][k] * l[n] + l[m] * dl[n][k]);
            dg[m][n][3] = 0;
        }
    T lu[4] = {l[0], l[1], l[2], -l[3]};
    T G1[4][4][4];
    for (int q_ = 0; q_ < 4; q_++)
        for (int m = 0; m < 4; m++)
            for (int n = 0; n < 4; n++) G1[q_][m][n] = (T)0.5 * (dg[q_][n][m] + dg[q_][m][n] - dg[m][n][q_]);
    T uu[4] = {u.x, u.y, u.z, u.w};
    T acc[4];
    for (int k = 0; k < 4; k++) {
        T s = 0;
        for (int m = 0; m < 4; m++)
            for (int n = 0; n < 4; n++) {
                T G = 0;
                for (int q_ = 0; q_ < 4; q_++) {
                    T gi = (k == q_ ? (k == 3 ? (T)-1 : (T)1) : (T)0) - f * lu[k] * lu[q_];
                    G += gi * G1[q_][m][n];
                }
                s += G * uu[m] * uu[n];
            }
        acc[k] = -s;
    }
    return {acc[0], acc[1], acc[2], acc[3]};
}

}  // namespace prr
