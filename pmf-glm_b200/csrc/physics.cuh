// Device-side ideal-MHD arithmetic for the B200 step kernels.
//
// Same scheme and operation order as the reference's precision-generic device functions
// (lib/MHDKernels/src/glm_physics.jl): cons2prim/prim2cons :11-23, fast_speed :24-27,
// phys_flux_x :28-34, rot_to/rot_flux_from :36-45 (here a compile-time axis permutation),
// MonCen/minmod :47-59, PPM :188-200, recon offsets :212-223, GLM pair :234-238,
// LLF/HLL :239-252, HLLD (Miyoshi & Kusano 2005) :255-307, riemann/riemann_ct :317-348.
// Compiled with fast math, as the reference's `@fastmath` kernels are.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pmf {

enum { RECON_PLM = 0, RECON_PPM = 1, RECON_PLM_MINMOD = 2 };
enum { RS_HLLD = 0, RS_HLL = 1, RS_LLF = 2 };
enum { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECT = 2 };

struct F9 {
  float v[9];
  __device__ __forceinline__ float& operator[](int i) { return v[i]; }
  __device__ __forceinline__ const float& operator[](int i) const { return v[i]; }
};

struct Phys {
  float gamma, smallr, pfl, llf_dmin, llf_pmin;
};

__device__ __forceinline__ F9 add9(const F9& a, const F9& b) {
  F9 r;
#pragma unroll
  for (int i = 0; i < 9; ++i) r[i] = a[i] + b[i];
  return r;
}
__device__ __forceinline__ F9 sub9(const F9& a, const F9& b) {
  F9 r;
#pragma unroll
  for (int i = 0; i < 9; ++i) r[i] = a[i] - b[i];
  return r;
}
__device__ __forceinline__ F9 neg9(const F9& a) {
  F9 r;
#pragma unroll
  for (int i = 0; i < 9; ++i) r[i] = -a[i];
  return r;
}

// conserved -> primitive with density and pressure floors (glm_physics.jl:11-18)
__device__ __forceinline__ F9 cons2prim(const F9& c, float g, float smallr, float pfl) {
  float rho = fmaxf(c[0], smallr);
  float ir = 1.0f / rho;
  float vx = c[1] * ir, vy = c[2] * ir, vz = c[3] * ir;
  float bx = c[5], by = c[6], bz = c[7];
  float ekin = 0.5f * (c[1] * c[1] + c[2] * c[2] + c[3] * c[3]) * ir;
  float emag = 0.5f * (bx * bx + by * by + bz * bz);
  float p = fmaxf((g - 1.0f) * (c[4] - ekin - emag), pfl);
  return F9{{rho, vx, vy, vz, p, bx, by, bz, c[8]}};
}

// primitive -> conserved (glm_physics.jl:19-23)
__device__ __forceinline__ F9 prim2cons(const F9& q, float g) {
  float rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4], bx = q[5], by = q[6], bz = q[7];
  float E = p / (g - 1.0f) + 0.5f * rho * (vx * vx + vy * vy + vz * vz) + 0.5f * (bx * bx + by * by + bz * bz);
  return F9{{rho, rho * vx, rho * vy, rho * vz, E, bx, by, bz, q[8]}};
}

// fast magnetosonic speed along the normal with normal field bn (glm_physics.jl:24-27)
__device__ __forceinline__ float fast_speed(const F9& q, float g, float bn) {
  float rho = q[0];
  float c2 = g * q[4] / rho;
  float b2 = (q[5] * q[5] + q[6] * q[6] + q[7] * q[7]) / rho;
  float d2 = 0.5f * (b2 + c2);
  return sqrtf(d2 + sqrtf(fmaxf(d2 * d2 - c2 * bn * bn / rho, 0.0f)));
}

// Axis permutations: D = 0, 1, 2 for x, y, z. rot_to maps the global (v, B) ordering to the
// frame whose first component is the D-normal; rot_back maps a flux back (glm_physics.jl:36-45).
template <int D> __device__ __forceinline__ F9 rot_to(const F9& q) {
  if (D == 0) return q;
  if (D == 1) return F9{{q[0], q[2], q[3], q[1], q[4], q[6], q[7], q[5], q[8]}};
  return F9{{q[0], q[3], q[1], q[2], q[4], q[7], q[5], q[6], q[8]}};
}
template <int D> __device__ __forceinline__ F9 rot_back(const F9& f) {
  if (D == 0) return f;
  if (D == 1) return F9{{f[0], f[3], f[1], f[2], f[4], f[7], f[5], f[6], f[8]}};
  return F9{{f[0], f[2], f[3], f[1], f[4], f[6], f[7], f[5], f[8]}};
}

// x-normal ideal-MHD flux; F[Bn] = F[psi] = 0 (glm_physics.jl:28-34)
__device__ __forceinline__ F9 phys_flux_x(const F9& q, float g) {
  float rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4], bx = q[5], by = q[6], bz = q[7];
  float b2 = bx * bx + by * by + bz * bz;
  float ptot = p + 0.5f * b2;
  float E = p / (g - 1.0f) + 0.5f * rho * (vx * vx + vy * vy + vz * vz) + 0.5f * b2;
  float vb = vx * bx + vy * by + vz * bz;
  return F9{{rho * vx, rho * vx * vx + ptot - bx * bx, rho * vx * vy - bx * by, rho * vx * vz - bx * bz,
             (E + ptot) * vx - bx * vb, 0.0f, vx * by - vy * bx, vx * bz - vz * bx, 0.0f}};
}
template <int D> __device__ __forceinline__ F9 dir_flux(const F9& q, float g) {
  return rot_back<D>(phys_flux_x(rot_to<D>(q), g));
}

// MonCen (slope_type 2) and minmod limiters (glm_physics.jl:47-59)
__device__ __forceinline__ float moncen(float dl, float dr) {
  float dc = 0.5f * (dl + dr);
  float sgn = dc >= 0.0f ? 1.0f : -1.0f;
  float val = sgn * fminf(2.0f * fminf(fabsf(dl), fabsf(dr)), fabsf(dc));
  return dl * dr <= 0.0f ? 0.0f : val;
}
__device__ __forceinline__ float minmod(float dl, float dr) {
  float sgn = dl >= 0.0f ? 1.0f : -1.0f;
  return dl * dr <= 0.0f ? 0.0f : sgn * fminf(fabsf(dl), fabsf(dr));
}
// local CW84 PPM edges, monotonised (glm_physics.jl:188-200)
__device__ __forceinline__ void ppm_edges(float qm, float q0, float qp, float& oL, float& oR) {
  float slope = (qp - qm) * 0.25f;
  float curve = (qm - 2.0f * q0 + qp) / 12.0f;
  float qL = q0 - slope + curve, qR = q0 + slope + curve, qa = q0;
  float dq = qR - qL, qmid = 0.5f * (qL + qR), dq2_6 = dq * dq / 6.0f, diff = (qa - qmid) * dq;
  if ((qR - qa) * (qa - qL) <= 0.0f) { oL = qa; oR = qa; }
  else if (diff > dq2_6) { oL = 3.0f * qa - 2.0f * qR; oR = qR; }
  else if (diff < -dq2_6) { oL = qL; oR = 3.0f * qa - 2.0f * qL; }
  else { oL = qL; oR = qR; }
}

// Per-axis face offsets about the cell mean. For the PLM limiters dL = -dR, so only dR is
// produced and dL is implied (glm_physics.jl:212-219); PPM produces both (:220-223).
template <int RECON> struct Offsets {
  F9 dR;
  __device__ __forceinline__ float l(int i) const { return -dR[i]; }
};
template <> struct Offsets<RECON_PPM> {
  F9 dL, dR;
  __device__ __forceinline__ float l(int i) const { return dL[i]; }
};

template <int RECON>
__device__ __forceinline__ Offsets<RECON> recon(const F9& mm, const F9& m0, const F9& mp) {
  Offsets<RECON> o;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    if constexpr (RECON == RECON_PLM) {
      o.dR[i] = 0.5f * moncen(m0[i] - mm[i], mp[i] - m0[i]);
    } else if constexpr (RECON == RECON_PLM_MINMOD) {
      o.dR[i] = 0.5f * minmod(m0[i] - mm[i], mp[i] - m0[i]);
    } else {
      float a, b;
      ppm_edges(mm[i], m0[i], mp[i], a, b);
      o.dL[i] = a - m0[i];
      o.dR[i] = b - m0[i];
    }
  }
  return o;
}
template <int RECON> __device__ __forceinline__ F9 face_lo(const F9& mh, const Offsets<RECON>& o) {
  F9 r;
#pragma unroll
  for (int i = 0; i < 9; ++i) r[i] = mh[i] + o.l(i);
  return r;
}
template <int RECON> __device__ __forceinline__ F9 face_hi(const F9& mh, const Offsets<RECON>& o) {
  F9 r;
#pragma unroll
  for (int i = 0; i < 9; ++i) r[i] = mh[i] + o.dR[i];
  return r;
}

// flux difference F(m0 + dR) - F(m0 + dL) along axis D (one term of the Hancock predictor)
template <int D, int RECON>
__device__ __forceinline__ F9 hancock_term(const F9& m0, const Offsets<RECON>& o, float g) {
  F9 p = face_hi<RECON>(m0, o), m = face_lo<RECON>(m0, o);
  return sub9(dir_flux<D>(p, g), dir_flux<D>(m, g));
}

// ---- Riemann solvers in the face-normal frame (x-normal after rot_to) -----------------
// LLF / Rusanov (glm_physics.jl:239-244)
__device__ __forceinline__ F9 llf_x(const F9& L, const F9& R, float g, float ch, float fbn, float fpsi) {
  F9 fL = phys_flux_x(L, g), fR = phys_flux_x(R, g), uL = prim2cons(L, g), uR = prim2cons(R, g);
  float smax = fmaxf(fmaxf(fabsf(L[1]) + fast_speed(L, g, L[5]), fabsf(R[1]) + fast_speed(R, g, R[5])), ch);
  F9 f;
#pragma unroll
  for (int i = 0; i < 9; ++i) f[i] = 0.5f * (fL[i] + fR[i]) - 0.5f * smax * (uR[i] - uL[i]);
  f[5] = fbn;
  f[8] = fpsi;
  return f;
}
// HLL (glm_physics.jl:245-252)
__device__ __forceinline__ F9 hll_x(const F9& L, const F9& R, float g, float bn, float fbn, float fpsi) {
  float cfL = fast_speed(L, g, bn), cfR = fast_speed(R, g, bn);
  float SL = fminf(fminf(L[1] - cfL, R[1] - cfR), 0.0f);
  float SR = fmaxf(fmaxf(L[1] + cfL, R[1] + cfR), 0.0f);
  F9 fL = phys_flux_x(L, g), fR = phys_flux_x(R, g), uL = prim2cons(L, g), uR = prim2cons(R, g);
  float invd = 1.0f / (SR - SL);
  F9 f;
#pragma unroll
  for (int i = 0; i < 9; ++i) f[i] = (SR * fL[i] - SL * fR[i] + SL * SR * (uR[i] - uL[i])) * invd;
  f[5] = fbn;
  f[8] = fpsi;
  return f;
}
// single-star transverse state (glm_physics.jl:255-263)
__device__ __forceinline__ void hlld_star(float d, float u, float v, float w, float by, float bz, float S, float bn,
                                          float SM, float& ov, float& ow, float& oby, float& obz) {
  float denK = d * (S - u) * (S - SM) - bn * bn;
  if (fabsf(denK) < 1e-12f) {
    ov = v; ow = w; oby = by; obz = bz;
  } else {
    float fac = bn * (SM - u) / denK;
    ov = v - by * fac;
    ow = w - bz * fac;
    oby = by * (d * (S - u) * (S - u) - bn * bn) / denK;
    obz = bz * (d * (S - u) * (S - u) - bn * bn) / denK;
  }
}
// HLLD, Miyoshi & Kusano 2005 (glm_physics.jl:264-307)
__device__ __forceinline__ F9 hlld_x(const F9& L, const F9& R, float g, float bn, float fbn, float fpsi) {
  const float dL = L[0], uL = L[1], vL = L[2], wL = L[3], pL = L[4], byL = L[6], bzL = L[7];
  const float dR = R[0], uR = R[1], vR = R[2], wR = R[3], pR = R[4], byR = R[6], bzR = R[7];
  float b2L = bn * bn + byL * byL + bzL * bzL, b2R = bn * bn + byR * byR + bzR * bzR;
  float ptL = pL + 0.5f * b2L, ptR = pR + 0.5f * b2R;
  float EL = pL / (g - 1.0f) + 0.5f * dL * (uL * uL + vL * vL + wL * wL) + 0.5f * b2L;
  float ER = pR / (g - 1.0f) + 0.5f * dR * (uR * uR + vR * vR + wR * wR) + 0.5f * b2R;
  float cfL = fast_speed(L, g, bn), cfR = fast_speed(R, g, bn);
  float SL = fminf(fminf(uL, uR) - fmaxf(cfL, cfR), 0.0f);
  float SR = fmaxf(fmaxf(uL, uR) + fmaxf(cfL, cfR), 0.0f);
  float den = (SR - uR) * dR - (SL - uL) * dL;
  float SM = ((SR - uR) * dR * uR - (SL - uL) * dL * uL - ptR + ptL) / den;
  float pts = ((SR - uR) * dR * ptL - (SL - uL) * dL * ptR + dL * dR * (SR - uR) * (SL - uL) * (uR - uL)) / den;
  float dLs = fmaxf(dL * (SL - uL) / (SL - SM), 1e-12f), dRs = fmaxf(dR * (SR - uR) / (SR - SM), 1e-12f);
  float sqdLs = sqrtf(dLs), sqdRs = sqrtf(dRs);
  float SLs = SM - fabsf(bn) / sqdLs, SRs = SM + fabsf(bn) / sqdRs;
  float vyLs, vzLs, byLs, bzLs, vyRs, vzRs, byRs, bzRs;
  hlld_star(dL, uL, vL, wL, byL, bzL, SL, bn, SM, vyLs, vzLs, byLs, bzLs);
  hlld_star(dR, uR, vR, wR, byR, bzR, SR, bn, SM, vyRs, vzRs, byRs, bzRs);
  float vdotbL = uL * bn + vL * byL + wL * bzL, vdotbLs = SM * bn + vyLs * byLs + vzLs * bzLs;
  float ELs = ((SL - uL) * EL - ptL * uL + pts * SM + bn * (vdotbL - vdotbLs)) / (SL - SM);
  float vdotbR = uR * bn + vR * byR + wR * bzR, vdotbRs = SM * bn + vyRs * byRs + vzRs * bzRs;
  float ERs = ((SR - uR) * ER - ptR * uR + pts * SM + bn * (vdotbR - vdotbRs)) / (SR - SM);
  float sgn = bn >= 0.0f ? 1.0f : -1.0f;
  float invsum = 1.0f / (sqdLs + sqdRs);
  float vyss = (sqdLs * vyLs + sqdRs * vyRs + (byRs - byLs) * sgn) * invsum;
  float vzss = (sqdLs * vzLs + sqdRs * vzRs + (bzRs - bzLs) * sgn) * invsum;
  float byss = (sqdLs * byRs + sqdRs * byLs + sqdLs * sqdRs * (vyRs - vyLs) * sgn) * invsum;
  float bzss = (sqdLs * bzRs + sqdRs * bzLs + sqdLs * sqdRs * (vzRs - vzLs) * sgn) * invsum;
  float vdotbss = SM * bn + vyss * byss + vzss * bzss;
  float ELss = ELs - sqdLs * (vdotbLs - vdotbss) * sgn;
  float ERss = ERs + sqdRs * (vdotbRs - vdotbss) * sgn;
  // Only the selected fan state is assembled: the four branches of glm_physics.jl:297-305.
  F9 f;
  if (SLs >= 0.0f) {
    F9 FL = phys_flux_x(F9{{dL, uL, vL, wL, pL, bn, byL, bzL, 0.0f}}, g);
    const float UL[8] = {dL, dL * uL, dL * vL, dL * wL, EL, bn, byL, bzL};
    const float ULs[8] = {dLs, dLs * SM, dLs * vyLs, dLs * vzLs, ELs, bn, byLs, bzLs};
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FL[i] + SL * (ULs[i] - UL[i]);
  } else if (SM >= 0.0f) {
    F9 FL = phys_flux_x(F9{{dL, uL, vL, wL, pL, bn, byL, bzL, 0.0f}}, g);
    const float UL[8] = {dL, dL * uL, dL * vL, dL * wL, EL, bn, byL, bzL};
    const float ULs[8] = {dLs, dLs * SM, dLs * vyLs, dLs * vzLs, ELs, bn, byLs, bzLs};
    const float ULss[8] = {dLs, dLs * SM, dLs * vyss, dLs * vzss, ELss, bn, byss, bzss};
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FL[i] + SLs * ULss[i] - (SLs - SL) * ULs[i] - SL * UL[i];
  } else if (SRs >= 0.0f) {
    F9 FR = phys_flux_x(F9{{dR, uR, vR, wR, pR, bn, byR, bzR, 0.0f}}, g);
    const float UR[8] = {dR, dR * uR, dR * vR, dR * wR, ER, bn, byR, bzR};
    const float URs[8] = {dRs, dRs * SM, dRs * vyRs, dRs * vzRs, ERs, bn, byRs, bzRs};
    const float URss[8] = {dRs, dRs * SM, dRs * vyss, dRs * vzss, ERss, bn, byss, bzss};
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FR[i] + SRs * URss[i] - (SRs - SR) * URs[i] - SR * UR[i];
  } else {
    F9 FR = phys_flux_x(F9{{dR, uR, vR, wR, pR, bn, byR, bzR, 0.0f}}, g);
    const float UR[8] = {dR, dR * uR, dR * vR, dR * wR, ER, bn, byR, bzR};
    const float URs[8] = {dRs, dRs * SM, dRs * vyRs, dRs * vzRs, ERs, bn, byRs, bzRs};
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FR[i] + SR * (URs[i] - UR[i]);
  }
  f[5] = fbn;
  f[8] = fpsi;
  return f;
}

// GLM Riemann problem on a D-normal face (glm_physics.jl:317-329): floors, Dedner pair,
// the selected solver (HLLD with the LLF fallback at low density/pressure), rotate back.
template <int D, int RSOL>
__device__ __forceinline__ F9 riemann_glm(const F9& Lq, const F9& Rq, float ch, const Phys& P) {
  F9 L = rot_to<D>(Lq), R = rot_to<D>(Rq);
  L[0] = fmaxf(L[0], P.smallr); L[4] = fmaxf(L[4], P.pfl);
  R[0] = fmaxf(R[0], P.smallr); R[4] = fmaxf(R[4], P.pfl);
  float bns = 0.5f * (L[5] + R[5]) - 0.5f * (R[8] - L[8]) / ch;
  float psis = 0.5f * (L[8] + R[8]) - 0.5f * ch * (R[5] - L[5]);
  float fbn = psis, fpsi = ch * ch * bns;
  L[5] = bns; R[5] = bns;
  F9 f;
  if constexpr (RSOL == RS_LLF) {
    f = llf_x(L, R, P.gamma, ch, fbn, fpsi);
  } else if constexpr (RSOL == RS_HLL) {
    f = hll_x(L, R, P.gamma, bns, fbn, fpsi);
  } else {
    bool uself = (P.llf_dmin > 0.0f && fminf(L[0], R[0]) < P.llf_dmin) ||
                 (P.llf_pmin > 0.0f && fminf(L[4], R[4]) < P.llf_pmin);
    if (uself) f = llf_x(L, R, P.gamma, ch, fbn, fpsi);
    else f = hlld_x(L, R, P.gamma, bns, fbn, fpsi);
  }
  return rot_back<D>(f);
}

// Constrained-transport Riemann problem (glm_physics.jl:336-348): the caller has put the
// staggered face value into both states' normal-B slot; no psi, ch = 0 in the LLF speed.
template <int D, int RSOL>
__device__ __forceinline__ F9 riemann_ct(const F9& Lq, const F9& Rq, const Phys& P) {
  F9 L = rot_to<D>(Lq), R = rot_to<D>(Rq);
  L[0] = fmaxf(L[0], P.smallr); L[4] = fmaxf(L[4], P.pfl); L[8] = 0.0f;
  R[0] = fmaxf(R[0], P.smallr); R[4] = fmaxf(R[4], P.pfl); R[5] = L[5]; R[8] = 0.0f;
  float bns = L[5];
  F9 f;
  if constexpr (RSOL == RS_LLF) {
    f = llf_x(L, R, P.gamma, 0.0f, 0.0f, 0.0f);
  } else if constexpr (RSOL == RS_HLL) {
    f = hll_x(L, R, P.gamma, bns, 0.0f, 0.0f);
  } else {
    bool uself = (P.llf_dmin > 0.0f && fminf(L[0], R[0]) < P.llf_dmin) ||
                 (P.llf_pmin > 0.0f && fminf(L[4], R[4]) < P.llf_pmin);
    if (uself) f = llf_x(L, R, P.gamma, 0.0f, 0.0f, 0.0f);
    else f = hlld_x(L, R, P.gamma, bns, 0.0f, 0.0f);
  }
  return rot_back<D>(f);
}

template <int D, int RSOL, bool CT>
__device__ __forceinline__ F9 riemann(const F9& L, const F9& R, float ch, const Phys& P) {
  if constexpr (CT) return riemann_ct<D, RSOL>(L, R, P);
  else return riemann_glm<D, RSOL>(L, R, ch, P);
}

// max over axes of |v_d| + c_f(B_d) of a conserved state (timestep.jl:4-14)
__device__ __forceinline__ float cell_wavespeed(const F9& u, const Phys& P) {
  F9 q = cons2prim(u, P.gamma, P.smallr, P.pfl);
  float sx = fabsf(q[1]) + fast_speed(q, P.gamma, q[5]);
  float sy = fabsf(q[2]) + fast_speed(q, P.gamma, q[6]);
  float sz = fabsf(q[3]) + fast_speed(q, P.gamma, q[7]);
  return fmaxf(sx, fmaxf(sy, sz));
}

// Kahan-compensated accumulation with a persistent remainder (glm_physics.jl:349-359).
// The fast-math build must not reassociate it, so the rounding steps are explicit.
__device__ __forceinline__ float comp_add(float x, float dx, float& r) {
  float inc = __fadd_rn(dx, r);
  float upd = __fadd_rn(x, inc);
  r = __fsub_rn(inc, __fsub_rn(upd, x));
  return upd;
}

// BC index map for a logical cell index (boundary.jl:161-175, 0-based): returns the source
// index; *flip = -1 where a reflecting wall mirrors the normal vector components.
__device__ __forceinline__ int bc_index(int i, int n, int code, float* flip) {
  *flip = 1.0f;
  if (code == BC_PERIODIC) {
    int r = i % n;
    return r < 0 ? r + n : r;
  }
  if (code == BC_OUTFLOW) return i < 0 ? 0 : (i >= n ? n - 1 : i);
  int r = i;
  if (i < 0) { *flip = -1.0f; r = -1 - i; }
  else if (i >= n) { *flip = -1.0f; r = 2 * n - 1 - i; }
  // an axis shorter than the 2-cell stencil mirrors past its far end: clamp
  return r < 0 ? 0 : (r >= n ? n - 1 : r);
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace pmf
