// Scalar FP32 restatement of the reference's device arithmetic, as a direct port would compile
// it (lib/MHDKernels/src/glm_physics.jl, compiled with fast math like its `@fastmath`
// functions): the MonCen slope in the reference's form (:47-53), the offsets (:212-215), the
// Hancock predictor with six separate directional fluxes (:225-231) and HLLD with both sides'
// single- and double-starred states assembled before the fan branch is chosen (:255-307).
// For the benchmark's plain port only (libpmfport.so); the library's step kernels use
// physics.cuh.
#pragma once
#include "../csrc/physics.cuh"

namespace pmf {
namespace refarith {

// MonCen (slope_type 2, glm_physics.jl:47-51) and the half slope of the PLM offsets
// (prim_slope :52-53, recon_offsets :212-215)
__device__ __forceinline__ float moncen_ref(float dl, float dr) {
  const float dc = 0.5f * (dl + dr);
  const float sgn = dc >= 0.0f ? 1.0f : -1.0f;
  const float v = sgn * fminf(2.0f * fminf(fabsf(dl), fabsf(dr)), fabsf(dc));
  return dl * dr <= 0.0f ? 0.0f : v;
}
__device__ __forceinline__ F9 plm_slope(const F9& mm, const F9& m0, const F9& mp) {
  F9 s;
#pragma unroll
  for (int i = 0; i < 9; ++i) s[i] = 0.5f * moncen_ref(m0[i] - mm[i], mp[i] - m0[i]);
  return s;
}

// hancock_edges (glm_physics.jl:225-231): six directional fluxes, one per face state
__device__ __forceinline__ F9 hancock_ref(const F9& m0, const F9& sx, const F9& sy, const F9& sz, float dtdx,
                                          float g) {
  const F9 u0 = prim2cons(m0, g);
  const float h = 0.5f * dtdx;
  F9 a, b;
#pragma unroll
  for (int i = 0; i < 9; ++i) { a[i] = m0[i] + sx[i]; b[i] = m0[i] - sx[i]; }
  const F9 fxp = dir_flux<0>(a, g), fxm = dir_flux<0>(b, g);
#pragma unroll
  for (int i = 0; i < 9; ++i) { a[i] = m0[i] + sy[i]; b[i] = m0[i] - sy[i]; }
  const F9 fyp = dir_flux<1>(a, g), fym = dir_flux<1>(b, g);
#pragma unroll
  for (int i = 0; i < 9; ++i) { a[i] = m0[i] + sz[i]; b[i] = m0[i] - sz[i]; }
  const F9 fzp = dir_flux<2>(a, g), fzm = dir_flux<2>(b, g);
  F9 r;
#pragma unroll
  for (int i = 0; i < 9; ++i) r[i] = u0[i] - h * (((fxp[i] - fxm[i]) + (fyp[i] - fym[i])) + (fzp[i] - fzm[i]));
  return r;
}

// _hlld_star (glm_physics.jl:255-263), with the degeneracy tolerance of Phys::dtol_rel
__device__ __forceinline__ void hlld_star_ref(float d, float u, float v, float w, float by, float bz, float S,
                                              float bn, float SM, float dtol_rel, float& vs, float& ws, float& bys,
                                              float& bzs) {
  const float denK = d * (S - u) * (S - SM) - bn * bn;
  if (fabsf(denK) < fmaxf(1e-12f, dtol_rel * bn * bn)) {
    vs = v; ws = w; bys = by; bzs = bz;
  } else {
    const float fac = bn * (SM - u) / denK;
    const float k = (d * (S - u) * (S - u) - bn * bn) / denK;
    vs = v - by * fac; ws = w - bz * fac; bys = by * k; bzs = bz * k;
  }
}

// hlld_x (glm_physics.jl:264-307), every state of both sides formed before the branch
__device__ __forceinline__ F9 hlld_ref(const F9& L, const F9& R, float g, float bn, float fbn, float fpsi,
                                       float dtol_rel) {
  const float dL = L[0], uL = L[1], vL = L[2], wL = L[3], pL = L[4], byL = L[6], bzL = L[7];
  const float dR = R[0], uR = R[1], vR = R[2], wR = R[3], pR = R[4], byR = R[6], bzR = R[7];
  const float b2L = bn * bn + byL * byL + bzL * bzL, b2R = bn * bn + byR * byR + bzR * bzR;
  const float ptL = pL + 0.5f * b2L, ptR = pR + 0.5f * b2R;
  const float EL = pL / (g - 1.0f) + 0.5f * dL * (uL * uL + vL * vL + wL * wL) + 0.5f * b2L;
  const float ER = pR / (g - 1.0f) + 0.5f * dR * (uR * uR + vR * vR + wR * wR) + 0.5f * b2R;
  const float cfL = fast_speed(L, g, bn), cfR = fast_speed(R, g, bn);
  const float SL = fminf(fminf(uL, uR) - fmaxf(cfL, cfR), 0.0f);
  const float SR = fmaxf(fmaxf(uL, uR) + fmaxf(cfL, cfR), 0.0f);
  const float UL[8] = {dL, dL * uL, dL * vL, dL * wL, EL, bn, byL, bzL};
  const float UR[8] = {dR, dR * uR, dR * vR, dR * wR, ER, bn, byR, bzR};
  const F9 FL = phys_flux_x(F9{{dL, uL, vL, wL, pL, bn, byL, bzL, 0.0f}}, g);
  const F9 FR = phys_flux_x(F9{{dR, uR, vR, wR, pR, bn, byR, bzR, 0.0f}}, g);
  const float den = (SR - uR) * dR - (SL - uL) * dL;
  const float SM = ((SR - uR) * dR * uR - (SL - uL) * dL * uL - ptR + ptL) / den;
  const float pts = ((SR - uR) * dR * ptL - (SL - uL) * dL * ptR + dL * dR * (SR - uR) * (SL - uL) * (uR - uL)) / den;
  const float dLs = fmaxf(dL * (SL - uL) / (SL - SM), 1e-12f), dRs = fmaxf(dR * (SR - uR) / (SR - SM), 1e-12f);
  const float sqdLs = sqrtf(dLs), sqdRs = sqrtf(dRs);
  const float SLs = SM - fabsf(bn) / sqdLs, SRs = SM + fabsf(bn) / sqdRs;
  float vyLs, vzLs, byLs, bzLs, vyRs, vzRs, byRs, bzRs;
  hlld_star_ref(dL, uL, vL, wL, byL, bzL, SL, bn, SM, dtol_rel, vyLs, vzLs, byLs, bzLs);
  hlld_star_ref(dR, uR, vR, wR, byR, bzR, SR, bn, SM, dtol_rel, vyRs, vzRs, byRs, bzRs);
  const float vdotbL = uL * bn + vL * byL + wL * bzL, vdotbLs = SM * bn + vyLs * byLs + vzLs * bzLs;
  const float ELs = ((SL - uL) * EL - ptL * uL + pts * SM + bn * (vdotbL - vdotbLs)) / (SL - SM);
  const float vdotbR = uR * bn + vR * byR + wR * bzR, vdotbRs = SM * bn + vyRs * byRs + vzRs * bzRs;
  const float ERs = ((SR - uR) * ER - ptR * uR + pts * SM + bn * (vdotbR - vdotbRs)) / (SR - SM);
  const float ULs[8] = {dLs, dLs * SM, dLs * vyLs, dLs * vzLs, ELs, bn, byLs, bzLs};
  const float URs[8] = {dRs, dRs * SM, dRs * vyRs, dRs * vzRs, ERs, bn, byRs, bzRs};
  const float sgn = bn >= 0.0f ? 1.0f : -1.0f, invsum = 1.0f / (sqdLs + sqdRs);
  const float vyss = (sqdLs * vyLs + sqdRs * vyRs + (byRs - byLs) * sgn) * invsum;
  const float vzss = (sqdLs * vzLs + sqdRs * vzRs + (bzRs - bzLs) * sgn) * invsum;
  const float byss = (sqdLs * byRs + sqdRs * byLs + sqdLs * sqdRs * (vyRs - vyLs) * sgn) * invsum;
  const float bzss = (sqdLs * bzRs + sqdRs * bzLs + sqdLs * sqdRs * (vzRs - vzLs) * sgn) * invsum;
  const float vdotbss = SM * bn + vyss * byss + vzss * bzss;
  const float ELss = ELs - sqdLs * (vdotbLs - vdotbss) * sgn, ERss = ERs + sqdRs * (vdotbRs - vdotbss) * sgn;
  const float ULss[8] = {dLs, dLs * SM, dLs * vyss, dLs * vzss, ELss, bn, byss, bzss};
  const float URss[8] = {dRs, dRs * SM, dRs * vyss, dRs * vzss, ERss, bn, byss, bzss};
  F9 f;
  if (SLs >= 0.0f) {
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FL[i] + SL * (ULs[i] - UL[i]);
  } else if (SM >= 0.0f) {
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FL[i] + SLs * ULss[i] - (SLs - SL) * ULs[i] - SL * UL[i];
  } else if (SRs >= 0.0f) {
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FR[i] + SRs * URss[i] - (SRs - SR) * URs[i] - SR * UR[i];
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FR[i] + SR * (URs[i] - UR[i]);
  }
  f[5] = fbn;
  f[8] = fpsi;
  return f;
}

// riemann (glm_physics.jl:317-329): floors, Dedner pair with a division by ch, LLF fallback,
// HLLD, rotation back
template <int D>
__device__ __forceinline__ F9 riemann_ref(const F9& Lq, const F9& Rq, float ch, const Phys& P) {
  F9 L = rot_to<D>(Lq), R = rot_to<D>(Rq);
  L[0] = fmaxf(L[0], P.smallr); L[4] = fmaxf(L[4], P.pfl);
  R[0] = fmaxf(R[0], P.smallr); R[4] = fmaxf(R[4], P.pfl);
  const float bns = 0.5f * (L[5] + R[5]) - 0.5f * (R[8] - L[8]) / ch;
  const float psis = 0.5f * (L[8] + R[8]) - 0.5f * ch * (R[5] - L[5]);
  const float fbn = psis, fpsi = ch * ch * bns;
  L[5] = bns; R[5] = bns;
  const bool uself = (P.llf_dmin > 0.0f && fminf(L[0], R[0]) < P.llf_dmin) ||
                     (P.llf_pmin > 0.0f && fminf(L[4], R[4]) < P.llf_pmin);
  const F9 f = uself ? llf_x(L, R, P.gamma, ch, fbn, fpsi) : hlld_ref(L, R, P.gamma, bns, fbn, fpsi, P.dtol_rel);
  return rot_back<D>(f);
}

}  // namespace refarith
}  // namespace pmf
