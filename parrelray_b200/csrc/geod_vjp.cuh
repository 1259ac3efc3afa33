// geod_vjp.cuh - reverse-mode derivative (vector-Jacobian product) of the
// Kerr-Schild geodesic acceleration geod_ks (prr_device.cuh, the FP64 form
// of the stepper): given weights w[4] on the outputs G = du/dlambda, returns
//   gx[k] = sum_r w_r dG_r/dx_k, gu[k] = sum_r w_r dG_r/du_k (k = x, y, z, t),
//   gM = sum_r w_r dG_r/dM,      ga = sum_r w_r dG_r/da.
// The adjoint of one stage of the RKF45 step needs exactly this product; one
// reverse sweep costs about three forward evaluations, where forward-mode
// dual numbers would carry ten tangents through every operation.
//
// The forward part repeats geod_ks operation for operation; the reverse part
// visits the same operations last to first (x_b denotes dOut/dx).  The time
// coordinate x^t does not enter the acceleration, so gx[3] = 0.
#pragma once
#include "prr_device.cuh"

namespace prr {

PRR_DEV void geod_vjp(const V4<double> &p, const V4<double> &u, double M, double a, const double w[4], double gx[4],
                      double gu[4], double &gM, double &ga)
{
    // ---- forward (as geod_ks<double, true>, the stepper's form) ----
    const double X = p.x, Y = p.y, Z = p.z;
    const double a2 = a * a;
    const double R2 = X * X + Y * Y + Z * Z;
    const double b = R2 - a2;
    const double S2 = b * b + 4.0 * a2 * Z * Z;
    const double iS = frsqrt<double>(S2), S = S2 * iS;
    const double r2 = 0.5 * (b + S);
    const double ir = frsqrt<double>(r2), r = r2 * ir;
    const double q = r2 + a2, iq = frcp<double>(q);
    const double Sig = r2 * r2 + a2 * Z * Z, iSig = frcp<double>(Sig);
    const double rS = r * iS;
    const double drx = X * rS, dry = Y * rS, drz = Z * q * iS * ir;
    const double f = 2.0 * M * r2 * r * iSig;
    const double inner = 3.0 * ir - 4.0 * r2 * r * iSig;
    const double c1 = f * inner;
    const double dfx = c1 * drx, dfy = c1 * dry, dfz = c1 * drz - 2.0 * f * a2 * Z * iSig;
    const double nlx = r * X + a * Y, nly = r * Y - a * X;
    const double lx = nlx * iq, ly = nly * iq, lz = Z * ir;
    const double ux = u.x, uy = u.y, uz = u.z, ut = u.w;
    const double Dr = ux * drx + uy * dry + uz * drz;
    const double Dq = 2.0 * r * Dr;
    const double nDlx = Dr * X + r * ux + a * uy - lx * Dq, nDly = Dr * Y + r * uy - a * ux - ly * Dq,
                 nDlz = uz - lz * Dr;
    const double Dlx = nDlx * iq, Dly = nDly * iq, Dlz = nDlz * ir;
    const double Df = ux * dfx + uy * dfy + uz * dfz;
    const double L = lx * ux + ly * uy + lz * uz + ut;
    const double DL = ux * Dlx + uy * Dly + uz * Dlz;
    const double ul = ux * lx + uy * ly;
    const double Pin = ux * X + uy * Y - 2.0 * r * ul;
    const double P = Pin * iq - uz * lz * ir;
    const double nLx = r * ux - a * uy, nLy = a * ux + r * uy;
    const double dLx = drx * P + nLx * iq, dLy = dry * P + nLy * iq, dLz = drz * P + uz * ir;
    const double A = L * Df + f * DL;
    const double fL = f * L, hL2 = 0.5 * L * L;
    const double Gx = lx * A + fL * Dlx - hL2 * dfx - fL * dLx;
    const double Gy = ly * A + fL * Dly - hL2 * dfy - fL * dLy;
    const double Gz = lz * A + fL * Dlz - hL2 * dfz - fL * dLz;
    const double Lam = lx * Gx + ly * Gy + lz * Gz - A;
    const double fLam = f * Lam;
    // outputs: fLam lx - Gx, fLam ly - Gy, fLam lz - Gz, A - fLam

    // ---- reverse ----
    const double w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
    double fLam_b = w0 * lx + w1 * ly + w2 * lz - w3;
    double lx_b = w0 * fLam, ly_b = w1 * fLam, lz_b = w2 * fLam;
    double Gx_b = -w0, Gy_b = -w1, Gz_b = -w2, A_b = w3;
    // fLam = f Lam
    double f_b = fLam_b * Lam;
    const double Lam_b = fLam_b * f;
    // Lam = lx Gx + ly Gy + lz Gz - A
    lx_b += Lam_b * Gx; Gx_b += Lam_b * lx;
    ly_b += Lam_b * Gy; Gy_b += Lam_b * ly;
    lz_b += Lam_b * Gz; Gz_b += Lam_b * lz;
    A_b -= Lam_b;
    // Gc = lc A + fL Dlc - hL2 dfc - fL dLc
    lx_b += Gx_b * A; ly_b += Gy_b * A; lz_b += Gz_b * A;
    A_b += Gx_b * lx + Gy_b * ly + Gz_b * lz;
    double fL_b = Gx_b * (Dlx - dLx) + Gy_b * (Dly - dLy) + Gz_b * (Dlz - dLz);
    double Dlx_b = Gx_b * fL, Dly_b = Gy_b * fL, Dlz_b = Gz_b * fL;
    const double hL2_b = -(Gx_b * dfx + Gy_b * dfy + Gz_b * dfz);
    double dfx_b = -Gx_b * hL2, dfy_b = -Gy_b * hL2, dfz_b = -Gz_b * hL2;
    const double dLx_b = -Gx_b * fL, dLy_b = -Gy_b * fL, dLz_b = -Gz_b * fL;
    // fL = f L, hL2 = L^2 / 2
    f_b += fL_b * L;
    double L_b = fL_b * f + hL2_b * L;
    // A = L Df + f DL
    L_b += A_b * Df;
    const double Df_b = A_b * L;
    f_b += A_b * DL;
    const double DL_b = A_b * f;
    // dLz = drz P + uz ir
    double drz_b = dLz_b * P;
    double P_b = dLz_b * drz;
    double uz_b = dLz_b * ir;
    double ir_b = dLz_b * uz;
    // dLy = dry P + (a ux + r uy) iq
    double dry_b = dLy_b * P;
    P_b += dLy_b * dry;
    double t = dLy_b * iq;
    double a_b = t * ux, ux_b = t * a, r_b = t * uy, uy_b = t * r;
    double iq_b = dLy_b * nLy;
    // dLx = drx P + (r ux - a uy) iq
    double drx_b = dLx_b * P;
    P_b += dLx_b * drx;
    t = dLx_b * iq;
    r_b += t * ux; ux_b += t * r; a_b -= t * uy; uy_b -= t * a;
    iq_b += dLx_b * nLx;
    // P = Pin iq - uz lz ir,  Pin = ux X + uy Y - 2 r (ux lx + uy ly)
    t = P_b * iq;
    iq_b += P_b * Pin;
    ux_b += t * (X - 2.0 * r * lx); uy_b += t * (Y - 2.0 * r * ly);
    double X_b = t * ux, Y_b = t * uy;
    r_b -= 2.0 * t * ul;
    lx_b -= 2.0 * t * r * ux; ly_b -= 2.0 * t * r * uy;
    uz_b -= P_b * lz * ir; lz_b -= P_b * uz * ir; ir_b -= P_b * uz * lz;
    // DL = ux Dlx + uy Dly + uz Dlz
    ux_b += DL_b * Dlx; Dlx_b += DL_b * ux;
    uy_b += DL_b * Dly; Dly_b += DL_b * uy;
    uz_b += DL_b * Dlz; Dlz_b += DL_b * uz;
    // L = lx ux + ly uy + lz uz + ut
    lx_b += L_b * ux; ux_b += L_b * lx;
    ly_b += L_b * uy; uy_b += L_b * ly;
    lz_b += L_b * uz; uz_b += L_b * lz;
    const double ut_b = L_b;
    // Df = ux dfx + uy dfy + uz dfz
    ux_b += Df_b * dfx; dfx_b += Df_b * ux;
    uy_b += Df_b * dfy; dfy_b += Df_b * uy;
    uz_b += Df_b * dfz; dfz_b += Df_b * uz;
    // Dlz = (uz - lz Dr) ir
    t = Dlz_b * ir;
    uz_b += t; lz_b -= t * Dr;
    double Dr_b = -t * lz;
    ir_b += Dlz_b * nDlz;
    // Dly = (Dr Y + r uy - a ux - ly Dq) iq
    t = Dly_b * iq;
    Dr_b += t * Y; Y_b += t * Dr; r_b += t * uy; uy_b += t * r; a_b -= t * ux; ux_b -= t * a; ly_b -= t * Dq;
    double Dq_b = -t * ly;
    iq_b += Dly_b * nDly;
    // Dlx = (Dr X + r ux + a uy - lx Dq) iq
    t = Dlx_b * iq;
    Dr_b += t * X; X_b += t * Dr; r_b += t * ux; ux_b += t * r; a_b += t * uy; uy_b += t * a; lx_b -= t * Dq;
    Dq_b -= t * lx;
    iq_b += Dlx_b * nDlx;
    // Dq = 2 r Dr
    r_b += 2.0 * Dq_b * Dr; Dr_b += 2.0 * Dq_b * r;
    // Dr = ux drx + uy dry + uz drz
    ux_b += Dr_b * drx; drx_b += Dr_b * ux;
    uy_b += Dr_b * dry; dry_b += Dr_b * uy;
    uz_b += Dr_b * drz; drz_b += Dr_b * uz;
    // lz = Z ir
    double Z_b = lz_b * ir;
    ir_b += lz_b * Z;
    // ly = (r Y - a X) iq
    t = ly_b * iq;
    r_b += t * Y; Y_b += t * r; a_b -= t * X; X_b -= t * a;
    iq_b += ly_b * nly;
    // lx = (r X + a Y) iq
    t = lx_b * iq;
    r_b += t * X; X_b += t * r; a_b += t * Y; Y_b += t * a;
    iq_b += lx_b * nlx;
    // dfz = c1 drz - 2 f a2 Z iSig
    double c1_b = dfz_b * drz;
    drz_b += dfz_b * c1;
    t = -2.0 * dfz_b;
    f_b += t * a2 * Z * iSig;
    double a2_b = t * f * Z * iSig;
    Z_b += t * f * a2 * iSig;
    double iSig_b = t * f * a2 * Z;
    // dfx = c1 drx, dfy = c1 dry
    c1_b += dfx_b * drx + dfy_b * dry;
    drx_b += dfx_b * c1; dry_b += dfy_b * c1;
    // c1 = f (3 ir - 4 r2 r iSig)
    f_b += c1_b * inner;
    t = c1_b * f;
    ir_b += 3.0 * t;
    double r2_b = -4.0 * t * r * iSig;
    r_b -= 4.0 * t * r2 * iSig;
    iSig_b -= 4.0 * t * r2 * r;
    // f = 2 M r2 r iSig
    gM = f_b * 2.0 * r2 * r * iSig;
    r2_b += f_b * 2.0 * M * r * iSig;
    r_b += f_b * 2.0 * M * r2 * iSig;
    iSig_b += f_b * 2.0 * M * r2 * r;
    // drz = Z q iS ir
    Z_b += drz_b * q * iS * ir;
    double q_b = drz_b * Z * iS * ir;
    double iS_b = drz_b * Z * q * ir;
    ir_b += drz_b * Z * q * iS;
    // drx = X rS, dry = Y rS
    X_b += drx_b * rS; Y_b += dry_b * rS;
    const double rS_b = drx_b * X + dry_b * Y;
    // rS = r iS
    r_b += rS_b * iS; iS_b += rS_b * r;
    // iSig = 1/Sig, Sig = r2^2 + a2 Z^2
    const double Sig_b = -iSig_b * iSig * iSig;
    r2_b += Sig_b * 2.0 * r2; a2_b += Sig_b * Z * Z; Z_b += Sig_b * 2.0 * a2 * Z;
    // iq = 1/q, q = r2 + a2
    q_b -= iq_b * iq * iq;
    r2_b += q_b; a2_b += q_b;
    // ir = 1/r, r = sqrt(r2)
    r_b -= ir_b * ir * ir;
    r2_b += r_b * 0.5 * ir;
    // r2 = (b + S)/2
    double b_b = 0.5 * r2_b;
    double S_b = 0.5 * r2_b;
    // iS = 1/S, S = sqrt(S2)
    S_b -= iS_b * iS * iS;
    const double S2_b = S_b * 0.5 * iS;
    // S2 = b^2 + 4 a2 Z^2
    b_b += S2_b * 2.0 * b; a2_b += S2_b * 4.0 * Z * Z; Z_b += S2_b * 8.0 * a2 * Z;
    // b = R2 - a2, R2 = X^2 + Y^2 + Z^2
    a2_b -= b_b;
    X_b += b_b * 2.0 * X; Y_b += b_b * 2.0 * Y; Z_b += b_b * 2.0 * Z;
    // a2 = a^2
    a_b += a2_b * 2.0 * a;

    gx[0] = X_b; gx[1] = Y_b; gx[2] = Z_b; gx[3] = 0.0;
    gu[0] = ux_b; gu[1] = uy_b; gu[2] = uz_b; gu[3] = ut_b;
    ga = a_b;
}

}  // namespace prr
