// CPU oracle for the PMFGLM ideal-MHD Godunov step — TEST INFRASTRUCTURE ONLY.
//
// This file is a plain C++ restatement (templated on float/double, OpenMP over cells)
// of the reference's portable per-cell MUSCL-Hancock GLM/CT scheme. It exists so the
// tests and the CPU-baseline leg of the benchmark can check the CUDA library against
// the reference algorithm; nothing in the shipped library links or calls it.
//
// Reference files followed (paths inside yipihey/pmf-glm):
//   lib/MHDKernels/src/glm_physics.jl   cons2prim/prim2cons :11-23, fast_speed :24-27,
//                                       phys_flux_x :28-34, rot_to/rot_flux_from :36-45,
//                                       moncen/minmod :47-59, PPM :188-200,
//                                       recon_offsets :212-223, hancock_edges :225-231,
//                                       glm_pair :234-238, llf_x/hll_x :239-252,
//                                       _hlld_star/hlld_x :255-307, riemann :317-329,
//                                       riemann_ct :336-348, _compensated_update! :349-359
//   lib/MHDKernels/src/integrator_ref.jl _mh_edges :17-26, per-cell body :69-160
//   lib/MHDKernels/src/boundary.jl       _bcidx :161-175, _loadU_bc :178-184
//   lib/MHDKernels/src/ct.jl             _ct_gs05 :57-66, _ct_emf_k! :71-93,
//                                       _ct_faceB[_comp]_k! :96-129, _ct_bcc_k! :132-143,
//                                       _ct_divb_face_k! :176-185, _ct_curl_k! :310-320,
//                                       _ct_cell_from_faces_k! :205-219
//   lib/MHDKernels/src/timestep.jl       _wavespeed_kernel! :4-14
//   lib/MHDKernels/src/diagnostics.jl    _divb_kernel! :6-20, conserved_totals :44-55
//
// Layout: every field array is SoA, nine (or three) contiguous blocks of nc = nx*ny*nz
// values, cell (i,j,k) (0-based) at ((k*ny)+j)*nx+i, x fastest — the reference's linidx.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <vector>

namespace {

enum { RECON_PLM = 0, RECON_PPM = 1, RECON_PLM_MINMOD = 2 };
enum { RS_HLLD = 0, RS_HLL = 1, RS_LLF = 2 };
enum { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECT = 2 };

template <class T> struct Q { T v[9]; T& operator[](int i) { return v[i]; } const T& operator[](int i) const { return v[i]; } };

template <class T> struct Phys {
  T gamma, smallr, pfl, llf_dmin, llf_pmin;
  int recon, rsol;
  // HLLD single-star degeneracy test |denK| < max(1e-12, dtol_rel * bn^2); dtol_rel = 0 is the
  // reference's own test |denK| < 1e-12 (glm_physics.jl:257)
  T dtol_rel;
};

// HLLD degeneracy census of one thread: solves, single-star sides with |denK| < 1e-12 (the
// reference's degenerate branch) and sides with 1e-12 <= |denK| < 1e-5 bn^2 (sent to the
// degenerate branch only by the relative test). Not part of the reference; a diagnostic.
struct Census {
  unsigned long long solves, ref_sides, rel_sides;
};

template <class T> inline T mx(T a, T b) { return a > b ? a : b; }
template <class T> inline T mn(T a, T b) { return a < b ? a : b; }

// glm_physics.jl:11-18
template <class T> Q<T> cons2prim(const Q<T>& c, T g, T smallr, T pfl) {
  T rho = mx(c[0], smallr); T ir = T(1) / rho;
  T vx = c[1] * ir, vy = c[2] * ir, vz = c[3] * ir, bx = c[5], by = c[6], bz = c[7];
  T ekin = T(0.5) * (c[1] * c[1] + c[2] * c[2] + c[3] * c[3]) * ir;
  T emag = T(0.5) * (bx * bx + by * by + bz * bz);
  T p = mx((g - T(1)) * (c[4] - ekin - emag), pfl);
  return Q<T>{{rho, vx, vy, vz, p, bx, by, bz, c[8]}};
}
// glm_physics.jl:19-23
template <class T> Q<T> prim2cons(const Q<T>& q, T g) {
  T rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4], bx = q[5], by = q[6], bz = q[7];
  T E = p / (g - T(1)) + T(0.5) * rho * (vx * vx + vy * vy + vz * vz) + T(0.5) * (bx * bx + by * by + bz * bz);
  return Q<T>{{rho, rho * vx, rho * vy, rho * vz, E, bx, by, bz, q[8]}};
}
// glm_physics.jl:24-27
template <class T> T fast_speed(const Q<T>& q, T g, T bn) {
  T rho = q[0]; T c2 = g * q[4] / rho;
  T b2 = (q[5] * q[5] + q[6] * q[6] + q[7] * q[7]) / rho; T d2 = T(0.5) * (b2 + c2);
  return std::sqrt(d2 + std::sqrt(mx(d2 * d2 - c2 * bn * bn / rho, T(0))));
}
// glm_physics.jl:28-34
template <class T> Q<T> phys_flux_x(const Q<T>& q, T g) {
  T rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4], bx = q[5], by = q[6], bz = q[7];
  T b2 = bx * bx + by * by + bz * bz; T ptot = p + T(0.5) * b2;
  T E = p / (g - T(1)) + T(0.5) * rho * (vx * vx + vy * vy + vz * vz) + T(0.5) * b2;
  T vb = vx * bx + vy * by + vz * bz;
  return Q<T>{{rho * vx, rho * vx * vx + ptot - bx * bx, rho * vx * vy - bx * by, rho * vx * vz - bx * bz,
               (E + ptot) * vx - bx * vb, T(0), vx * by - vy * bx, vx * bz - vz * bx, T(0)}};
}
// glm_physics.jl:36-45 (dir 0,1,2 = x,y,z)
template <class T> Q<T> rot_to(const Q<T>& q, int d) {
  if (d == 0) return q;
  if (d == 1) return Q<T>{{q[0], q[2], q[3], q[1], q[4], q[6], q[7], q[5], q[8]}};
  return Q<T>{{q[0], q[3], q[1], q[2], q[4], q[7], q[5], q[6], q[8]}};
}
template <class T> Q<T> rot_flux_from(const Q<T>& f, int d) {
  if (d == 0) return f;
  if (d == 1) return Q<T>{{f[0], f[3], f[1], f[2], f[4], f[7], f[5], f[6], f[8]}};
  return Q<T>{{f[0], f[2], f[3], f[1], f[4], f[6], f[7], f[5], f[8]}};
}
template <class T> Q<T> dir_flux(const Q<T>& q, int d, T g) { return rot_flux_from(phys_flux_x(rot_to(q, d), g), d); }

// glm_physics.jl:47-59
template <class T> T moncen(T dl, T dr) {
  T dc = T(0.5) * (dl + dr); T sgn = dc >= T(0) ? T(1) : T(-1);
  T val = sgn * mn(T(2) * mn(std::fabs(dl), std::fabs(dr)), std::fabs(dc));
  return dl * dr <= T(0) ? T(0) : val;
}
template <class T> T minmod(T dl, T dr) {
  T sgn = dl >= T(0) ? T(1) : T(-1);
  return dl * dr <= T(0) ? T(0) : sgn * mn(std::fabs(dl), std::fabs(dr));
}
// glm_physics.jl:188-200
template <class T> void ppm_edges(T qm, T q0, T qp, T& oL, T& oR) {
  T slope = (qp - qm) * T(0.25); T curve = (qm - T(2) * q0 + qp) / T(12);
  T qL = q0 - slope + curve, qR = q0 + slope + curve, qa = q0;
  T dq = qR - qL; T qmid = T(0.5) * (qL + qR); T dq2_6 = dq * dq / T(6); T diff = (qa - qmid) * dq;
  if ((qR - qa) * (qa - qL) <= T(0)) { oL = qa; oR = qa; }
  else if (diff > dq2_6) { oL = T(3) * qa - T(2) * qR; oR = qR; }
  else if (diff < -dq2_6) { oL = qL; oR = T(3) * qa - T(2) * qL; }
  else { oL = qL; oR = qR; }
}
// glm_physics.jl:212-223: per-axis face offsets (dL, dR) about the cell mean
template <class T> void recon_offsets(const Q<T>& mm, const Q<T>& m0, const Q<T>& mp, int rec, Q<T>& dL, Q<T>& dR) {
  for (int i = 0; i < 9; ++i) {
    if (rec == RECON_PLM) { T s = T(0.5) * moncen(m0[i] - mm[i], mp[i] - m0[i]); dL[i] = -s; dR[i] = s; }
    else if (rec == RECON_PLM_MINMOD) { T s = T(0.5) * minmod(m0[i] - mm[i], mp[i] - m0[i]); dL[i] = -s; dR[i] = s; }
    else { T a, b; ppm_edges(mm[i], m0[i], mp[i], a, b); dL[i] = a - m0[i]; dR[i] = b - m0[i]; }
  }
}
template <class T> Q<T> qadd(const Q<T>& a, const Q<T>& b) { Q<T> r; for (int i = 0; i < 9; ++i) r[i] = a[i] + b[i]; return r; }

// glm_physics.jl:225-231
template <class T> Q<T> hancock_edges(const Q<T>& m0, const Q<T>* dL, const Q<T>* dR, T dtdx, T g) {
  Q<T> u0 = prim2cons(m0, g); T h = T(0.5) * dtdx;
  Q<T> fp[3], fm[3];
  for (int d = 0; d < 3; ++d) { fp[d] = dir_flux(qadd(m0, dR[d]), d, g); fm[d] = dir_flux(qadd(m0, dL[d]), d, g); }
  Q<T> r;
  for (int i = 0; i < 9; ++i) r[i] = u0[i] - h * (((fp[0][i] - fm[0][i]) + (fp[1][i] - fm[1][i])) + (fp[2][i] - fm[2][i]));
  return r;
}

// glm_physics.jl:239-252
template <class T> Q<T> llf_x(const Q<T>& L, const Q<T>& R, T g, T ch, T fbn, T fpsi) {
  Q<T> fL = phys_flux_x(L, g), fR = phys_flux_x(R, g), uL = prim2cons(L, g), uR = prim2cons(R, g);
  T smax = mx(mx(std::fabs(L[1]) + fast_speed(L, g, L[5]), std::fabs(R[1]) + fast_speed(R, g, R[5])), ch);
  Q<T> f; for (int i = 0; i < 9; ++i) f[i] = T(0.5) * (fL[i] + fR[i]) - T(0.5) * smax * (uR[i] - uL[i]);
  f[5] = fbn; f[8] = fpsi; return f;
}
template <class T> Q<T> hll_x(const Q<T>& L, const Q<T>& R, T g, T bn, T fbn, T fpsi) {
  T cfL = fast_speed(L, g, bn), cfR = fast_speed(R, g, bn);
  T SL = mn(mn(L[1] - cfL, R[1] - cfR), T(0)); T SR = mx(mx(L[1] + cfL, R[1] + cfR), T(0));
  Q<T> fL = phys_flux_x(L, g), fR = phys_flux_x(R, g), uL = prim2cons(L, g), uR = prim2cons(R, g);
  T invd = T(1) / (SR - SL);
  Q<T> f; for (int i = 0; i < 9; ++i) f[i] = (SR * fL[i] - SL * fR[i] + SL * SR * (uR[i] - uL[i])) * invd;
  f[5] = fbn; f[8] = fpsi; return f;
}
// glm_physics.jl:255-263
template <class T> void hlld_star(T d, T u, T v, T w, T by, T bz, T S, T bn, T SM, T dtol_rel, T& ov, T& ow, T& oby,
                                  T& obz, Census* cen) {
  T denK = d * (S - u) * (S - SM) - bn * bn;
  // The reference's degeneracy test is |denK| < 1e-12 (dtol_rel = 0). With dtol_rel = 1e-5 it
  // is widened to |denK| < max(1e-12, 1e-5 bn^2), the FP32 rounding level of denK (a difference
  // of two terms of size bn^2), as the device solver's relative mode does: below it the
  // single-star states are ~1/denK and the fan flux hinges on a 1-ulp cancellation.
  if (cen) {
    const T a = std::fabs(denK);
    cen->ref_sides += a < T(1e-12);
    cen->rel_sides += a >= T(1e-12) && a < T(1e-5) * bn * bn;
  }
  if (std::fabs(denK) < mx(T(1e-12), dtol_rel * bn * bn)) { ov = v; ow = w; oby = by; obz = bz; return; }
  T fac = bn * (SM - u) / denK;
  ov = v - by * fac; ow = w - bz * fac;
  oby = by * (d * (S - u) * (S - u) - bn * bn) / denK;
  obz = bz * (d * (S - u) * (S - u) - bn * bn) / denK;
}
// glm_physics.jl:264-307
template <class T> Q<T> hlld_x(const Q<T>& L, const Q<T>& R, T g, T bn, T fbn, T fpsi, T dtol_rel,
                               Census* cen = nullptr) {
  if (cen) cen->solves += 1;
  T dL = L[0], uL = L[1], vL = L[2], wL = L[3], pL = L[4], byL = L[6], bzL = L[7];
  T dR = R[0], uR = R[1], vR = R[2], wR = R[3], pR = R[4], byR = R[6], bzR = R[7];
  T b2L = bn * bn + byL * byL + bzL * bzL, b2R = bn * bn + byR * byR + bzR * bzR;
  T ptL = pL + T(0.5) * b2L, ptR = pR + T(0.5) * b2R;
  T EL = pL / (g - T(1)) + T(0.5) * dL * (uL * uL + vL * vL + wL * wL) + T(0.5) * b2L;
  T ER = pR / (g - T(1)) + T(0.5) * dR * (uR * uR + vR * vR + wR * wR) + T(0.5) * b2R;
  T cfL = fast_speed(L, g, bn), cfR = fast_speed(R, g, bn);
  T SL = mn(mn(uL, uR) - mx(cfL, cfR), T(0)); T SR = mx(mx(uL, uR) + mx(cfL, cfR), T(0));
  Q<T> UL{{dL, dL * uL, dL * vL, dL * wL, EL, bn, byL, bzL, T(0)}};
  Q<T> UR{{dR, dR * uR, dR * vR, dR * wR, ER, bn, byR, bzR, T(0)}};
  Q<T> FL = phys_flux_x(Q<T>{{dL, uL, vL, wL, pL, bn, byL, bzL, T(0)}}, g);
  Q<T> FR = phys_flux_x(Q<T>{{dR, uR, vR, wR, pR, bn, byR, bzR, T(0)}}, g);
  T den = (SR - uR) * dR - (SL - uL) * dL;
  T SM = ((SR - uR) * dR * uR - (SL - uL) * dL * uL - ptR + ptL) / den;
  T pts = ((SR - uR) * dR * ptL - (SL - uL) * dL * ptR + dL * dR * (SR - uR) * (SL - uL) * (uR - uL)) / den;
  T dLs = mx(dL * (SL - uL) / (SL - SM), T(1e-12)), dRs = mx(dR * (SR - uR) / (SR - SM), T(1e-12));
  T sqdLs = std::sqrt(dLs), sqdRs = std::sqrt(dRs);
  T SLs = SM - std::fabs(bn) / sqdLs, SRs = SM + std::fabs(bn) / sqdRs;
  T vyLs, vzLs, byLs, bzLs, vyRs, vzRs, byRs, bzRs;
  hlld_star(dL, uL, vL, wL, byL, bzL, SL, bn, SM, dtol_rel, vyLs, vzLs, byLs, bzLs, cen);
  hlld_star(dR, uR, vR, wR, byR, bzR, SR, bn, SM, dtol_rel, vyRs, vzRs, byRs, bzRs, cen);
  T vdotbL = uL * bn + vL * byL + wL * bzL, vdotbLs = SM * bn + vyLs * byLs + vzLs * bzLs;
  T ELs = ((SL - uL) * EL - ptL * uL + pts * SM + bn * (vdotbL - vdotbLs)) / (SL - SM);
  T vdotbR = uR * bn + vR * byR + wR * bzR, vdotbRs = SM * bn + vyRs * byRs + vzRs * bzRs;
  T ERs = ((SR - uR) * ER - ptR * uR + pts * SM + bn * (vdotbR - vdotbRs)) / (SR - SM);
  Q<T> ULs{{dLs, dLs * SM, dLs * vyLs, dLs * vzLs, ELs, bn, byLs, bzLs, T(0)}};
  Q<T> URs{{dRs, dRs * SM, dRs * vyRs, dRs * vzRs, ERs, bn, byRs, bzRs, T(0)}};
  T sgn = bn >= T(0) ? T(1) : T(-1); T invsum = T(1) / (sqdLs + sqdRs);
  T vyss = (sqdLs * vyLs + sqdRs * vyRs + (byRs - byLs) * sgn) * invsum;
  T vzss = (sqdLs * vzLs + sqdRs * vzRs + (bzRs - bzLs) * sgn) * invsum;
  T byss = (sqdLs * byRs + sqdRs * byLs + sqdLs * sqdRs * (vyRs - vyLs) * sgn) * invsum;
  T bzss = (sqdLs * bzRs + sqdRs * bzLs + sqdLs * sqdRs * (vzRs - vzLs) * sgn) * invsum;
  T vdotbss = SM * bn + vyss * byss + vzss * bzss;
  T ELss = ELs - sqdLs * (vdotbLs - vdotbss) * sgn, ERss = ERs + sqdRs * (vdotbRs - vdotbss) * sgn;
  Q<T> ULss{{dLs, dLs * SM, dLs * vyss, dLs * vzss, ELss, bn, byss, bzss, T(0)}};
  Q<T> URss{{dRs, dRs * SM, dRs * vyss, dRs * vzss, ERss, bn, byss, bzss, T(0)}};
  Q<T> f;
  if (SLs >= T(0)) { for (int i = 0; i < 9; ++i) f[i] = FL[i] + SL * (ULs[i] - UL[i]); }
  else if (SM >= T(0)) { for (int i = 0; i < 9; ++i) f[i] = FL[i] + SLs * ULss[i] - (SLs - SL) * ULs[i] - SL * UL[i]; }
  else if (SRs >= T(0)) { for (int i = 0; i < 9; ++i) f[i] = FR[i] + SRs * URss[i] - (SRs - SR) * URs[i] - SR * UR[i]; }
  else { for (int i = 0; i < 9; ++i) f[i] = FR[i] + SR * (URs[i] - UR[i]); }
  f[5] = fbn; f[8] = fpsi; return f;
}
// glm_physics.jl:317-329
// force_llf: LLF on this face whatever P.rsol, the masked fallback of the cube kernel
// (_cube_masked_riemann, integrator_cube.jl:68-79)
template <class T> Q<T> riemann(const Q<T>& Lq, const Q<T>& Rq, int d, T ch, const Phys<T>& P, Census* cen = nullptr,
                                bool force_llf = false) {
  Q<T> L = rot_to(Lq, d), R = rot_to(Rq, d);
  L[0] = mx(L[0], P.smallr); L[4] = mx(L[4], P.pfl);
  R[0] = mx(R[0], P.smallr); R[4] = mx(R[4], P.pfl);
  T bns = T(0.5) * (L[5] + R[5]) - T(0.5) * (R[8] - L[8]) / ch;
  T psis = T(0.5) * (L[8] + R[8]) - T(0.5) * ch * (R[5] - L[5]);
  T fbn = psis, fpsi = ch * ch * bns;
  L[5] = bns; R[5] = bns;
  bool uself = (P.llf_dmin > T(0) && mn(L[0], R[0]) < P.llf_dmin) || (P.llf_pmin > T(0) && mn(L[4], R[4]) < P.llf_pmin);
  Q<T> f;
  if (P.rsol == RS_LLF || force_llf) f = llf_x(L, R, P.gamma, ch, fbn, fpsi);
  else if (P.rsol == RS_HLL) f = hll_x(L, R, P.gamma, bns, fbn, fpsi);
  else f = uself ? llf_x(L, R, P.gamma, ch, fbn, fpsi) : hlld_x(L, R, P.gamma, bns, fbn, fpsi, P.dtol_rel, cen);
  return rot_flux_from(f, d);
}
// glm_physics.jl:336-348
template <class T> Q<T> riemann_ct(const Q<T>& Lq, const Q<T>& Rq, int d, const Phys<T>& P, Census* cen = nullptr,
                                   bool force_llf = false) {
  Q<T> L0 = rot_to(Lq, d), R0 = rot_to(Rq, d);
  Q<T> L = L0, R = R0;
  L[0] = mx(L0[0], P.smallr); L[4] = mx(L0[4], P.pfl); L[8] = T(0);
  R[0] = mx(R0[0], P.smallr); R[4] = mx(R0[4], P.pfl); R[5] = L0[5]; R[8] = T(0);
  T bns = L[5]; T z = T(0);
  bool uself = (P.llf_dmin > z && mn(L[0], R[0]) < P.llf_dmin) || (P.llf_pmin > z && mn(L[4], R[4]) < P.llf_pmin);
  Q<T> f;
  if (P.rsol == RS_LLF || force_llf) f = llf_x(L, R, P.gamma, z, z, z);
  else if (P.rsol == RS_HLL) f = hll_x(L, R, P.gamma, bns, z, z);
  else f = uself ? llf_x(L, R, P.gamma, z, z, z) : hlld_x(L, R, P.gamma, bns, z, z, P.dtol_rel, cen);
  return rot_flux_from(f, d);
}

// zlo/zhi: the planes a Godunov step updates (zhi <= zlo: all of them)
struct Grid { int nx, ny, nz, bc[3]; int zlo = 0, zhi = 0; };

// boundary.jl:161-175 (0-based)
inline void bcidx(int i, int n, int code, int& ii, int& flip) {
  flip = 1;
  if (code == BC_PERIODIC) { ii = ((i % n) + n) % n; return; }
  if (code == BC_OUTFLOW) { ii = i < 0 ? 0 : (i >= n ? n - 1 : i); return; }
  if (i < 0) { ii = -1 - i; flip = -1; }
  else if (i >= n) { ii = 2 * n - 1 - i; flip = -1; }
  else ii = i;
  ii = ii < 0 ? 0 : (ii >= n ? n - 1 : ii);  // axis shorter than the stencil
}
inline long lin(const Grid& g, int i, int j, int k) { return ((long)k * g.ny + j) * g.nx + i; }
inline long per(const Grid& g, int i, int j, int k) {
  i = ((i % g.nx) + g.nx) % g.nx; j = ((j % g.ny) + g.ny) % g.ny; k = ((k % g.nz) + g.nz) % g.nz;
  return lin(g, i, j, k);
}

// boundary.jl:178-187: conserved state under the per-axis BCs, as primitives
template <class T> Q<T> loadP(const Grid& g, const T* U, long nc, int i, int j, int k, const Phys<T>& P) {
  int ii, jj, kk, fx, fy, fz;
  bcidx(i, g.nx, g.bc[0], ii, fx); bcidx(j, g.ny, g.bc[1], jj, fy); bcidx(k, g.nz, g.bc[2], kk, fz);
  long c = lin(g, ii, jj, kk);
  Q<T> u{{U[c], U[nc + c] * T(fx), U[2 * nc + c] * T(fy), U[3 * nc + c] * T(fz), U[4 * nc + c],
          U[5 * nc + c] * T(fx), U[6 * nc + c] * T(fy), U[7 * nc + c] * T(fz), U[8 * nc + c]}};
  return cons2prim(u, P.gamma, P.smallr, P.pfl);
}

// integrator_ref.jl:17-26 — a cell's Hancock-predicted primitive and its per-axis offsets.
// first_order: zero offsets, the piecewise-constant states of the cube kernel's global
// fallback (CHECK == 3, integrator_cube.jl:168-177).
template <class T> struct Edges { Q<T> m0, mh, dL[3], dR[3]; };
template <class T> Edges<T> mh_edges(const Grid& g, const T* U, long nc, int i, int j, int k, T dtdx, const Phys<T>& P,
                                     bool first_order = false) {
  Edges<T> e;
  e.m0 = loadP(g, U, nc, i, j, k, P);
  if (first_order) {
    for (int d = 0; d < 3; ++d)
      for (int v = 0; v < 9; ++v) e.dL[d][v] = e.dR[d][v] = T(0);
  } else {
    recon_offsets(loadP(g, U, nc, i - 1, j, k, P), e.m0, loadP(g, U, nc, i + 1, j, k, P), P.recon, e.dL[0], e.dR[0]);
    recon_offsets(loadP(g, U, nc, i, j - 1, k, P), e.m0, loadP(g, U, nc, i, j + 1, k, P), P.recon, e.dL[1], e.dR[1]);
    recon_offsets(loadP(g, U, nc, i, j, k - 1, P), e.m0, loadP(g, U, nc, i, j, k + 1, P), P.recon, e.dL[2], e.dR[2]);
  }
  Q<T> uh = hancock_edges(e.m0, e.dL, e.dR, dtdx, P.gamma);
  e.mh = cons2prim(uh, P.gamma, P.smallr, P.pfl);
  return e;
}

// glm_physics.jl:349-359 (Kahan with a persistent per-cell remainder)
template <class T> T comp_update(T* r, long idx, T x, T dx) {
  T carry = r[idx]; T inc = dx + carry; T upd = x + inc;
  volatile T diff = upd - x;  // keep the compensation from being folded away
  r[idx] = inc - diff;
  return upd;
}

// ---- linear (Compton) drag toward a target velocity (glm_physics.jl:63-172) ------------
template <class T> T drag_phi1(T q) { return std::fabs(q) < T(1e-4) ? T(1) - q / T(2) + q * q / T(6) : -std::expm1(-q) / q; }
template <class T> void drag_work_coefficients(T q, T& A, T& C, T& D) {
  if (q < T(0.05)) {
    T q2 = q * q, q3 = q2 * q, q4 = q3 * q;
    A = q * (T(1) - q + T(2.0 / 3.0) * q2 - T(1.0 / 3.0) * q3 + T(2.0 / 15.0) * q4);
    C = q * (T(1) - q + T(7.0 / 12.0) * q2 - T(1.0 / 4.0) * q3 + T(31.0 / 360.0) * q4);
    D = q * (T(1.0 / 3.0) - q / T(4) + T(7.0 / 60.0) * q2 - q3 / T(24) + T(31.0 / 2520.0) * q4);
    return;
  }
  T em1 = -std::expm1(-q), em2 = -std::expm1(-T(2) * q);
  A = T(0.5) * em2;
  C = em1 * em1 / q;
  D = (q - T(2) * em1 + T(0.5) * em2) / (q * q);
}
template <class T> struct Drag {
  bool on;
  T qh, q;     // half-step and full-step impulse
  T v0[3];     // target velocity
};
// exact constant-force propagation of a face prediction (glm_physics.jl:71-84)
template <class T> Q<T> drag_predict_face(const Q<T>& q0, const Q<T>& qh, T impulse, const T* v0) {
  T decay = std::exp(-impulse), phi1 = drag_phi1(impulse);
  Q<T> r = qh;
  for (int c = 0; c < 3; ++c) r[1 + c] = v0[c] + decay * (q0[1 + c] - v0[c]) + phi1 * (qh[1 + c] - q0[1 + c]);
  return r;
}
// cell corrector: exact momentum response and integrated drag work (glm_physics.jl:128-172);
// the state with E still the trial's, the work qwork and the energy floor emin
// (`_drag_correct_conserved_parts`)
template <class T> Q<T> drag_correct_parts(const Q<T>& u0, const Q<T>& trial, T impulse, const T* v0, T smallr,
                                           T smallE, T& qwork_out, T& emin_out) {
  T decay = std::exp(-impulse), phi1 = drag_phi1(impulse), A, C, D;
  drag_work_coefficients(impulse, A, C, D);
  T rn = mx(trial[0], smallr), ro = mx(u0[0], smallr);
  T vo[3] = {u0[1] / ro, u0[2] / ro, u0[3] / ro};
  T vt[3] = {trial[1] / rn, trial[2] / rn, trial[3] / rn};
  T dv[3], w[3], vn[3], iw[3];
  for (int c = 0; c < 3; ++c) {
    dv[c] = vt[c] - vo[c];
    w[c] = vo[c] - v0[c];
    vn[c] = v0[c] + decay * w[c] + phi1 * dv[c];
    iw[c] = (T(1) - decay) * w[c] + (T(1) - phi1) * dv[c];
  }
  T w2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  T wdv = w[0] * dv[0] + w[1] * dv[1] + w[2] * dv[2];
  T dv2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
  T qwork = rn * (A * w2 + C * wdv + D * dv2 + v0[0] * iw[0] + v0[1] * iw[1] + v0[2] * iw[2]);
  T nm[3] = {rn * vn[0], rn * vn[1], rn * vn[2]};
  T ek = T(0.5) * (nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]) / rn;
  T eb = T(0.5) * (trial[5] * trial[5] + trial[6] * trial[6] + trial[7] * trial[7]);
  qwork_out = qwork;
  emin_out = ek + eb + smallE;
  return Q<T>{{rn, nm[0], nm[1], nm[2], trial[4], trial[5], trial[6], trial[7], trial[8]}};
}
template <class T> Q<T> drag_correct_conserved(const Q<T>& u0, const Q<T>& trial, T impulse, const T* v0, T smallr,
                                               T smallE) {
  T qwork, emin;
  Q<T> r = drag_correct_parts(u0, trial, impulse, v0, smallr, smallE, qwork, emin);
  r[4] = mx(trial[4] - qwork, emin);
  return r;
}

// ---- radiation-coupled step flags (integrator_ref.jl:33-39,140-156; integrator_cube.jl:85-124) ----
// corr is the packed 9*nc correction buffer: slot 0 is psi (read instead of U[8]), slots 1-3
// the velocity corrections added to every face state, slot 4 the accumulated density
// increment (track_density), slots 5-7 the Kahan remainders of cell B (track_magnetic,
// GLM only) and slot 8 that of E (track_energy).
// RAD_MASKED: the cube kernel's masked fallback (CHECK == 2, integrator_cube.jl:68-83,168-171):
// a cell whose mask entry is positive takes zero offsets, and a face with such a cell on either
// side takes LLF. The mask is slot 4 as it was before the step (`mask` holds that copy: the
// density increments of the same step land in slot 4).
enum { RAD_TRACK_DENSITY = 1, RAD_TRACK_MAGNETIC = 2, RAD_TRACK_ENERGY = 4, RAD_CHECK = 8, RAD_FIRST_ORDER = 16,
       RAD_MASKED = 32 };
template <class T> struct Rad {
  T* corr;   // null: no radiation coupling
  int flags;
  const T* mask = nullptr;  // RAD_MASKED: the per-cell mask
};
// integrator_cube.jl:108-124
template <class T> bool inadmissible(const Q<T>& r, const Phys<T>& P) {
  T gate = mx(P.smallr, P.llf_dmin);
  T ir = T(1) / mx(r[0], P.smallr);
  T ek = T(0.5) * (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) * ir;
  T eb = T(0.5) * (r[5] * r[5] + r[6] * r[6] + r[7] * r[7]);
  T eint = r[4] - ek - eb;
  T emin = P.pfl / (P.gamma - T(1));
  bool finite = std::isfinite(r[0]) && std::isfinite(eint);
  for (int v = 1; v < 9; ++v) finite = finite && std::isfinite(r[v]);
  return !finite || r[0] < gate || eint < emin;
}

// CT workspace slots (ct.jl:71-93 consumer order; state.jl:44-52 names)
enum { W_MFX = 0, W_MFY, W_MFZ, W_FXBY, W_FXBZ, W_FYBX, W_FYBZ, W_FZBX, W_FZBY, W_ECX, W_ECY, W_ECZ, W_EX, W_EY, W_EZ, W_N };

// integrator_ref.jl:69-160 — one Godunov step for every cell.
//   U (9nc) in, Un (9nc) out. resid: NULL or 7nc remainders (mx,my,mz,E,Bx,By,Bz).
//   CT: faces (3nc, lower-face normal B) and work (W_N*nc) non-NULL.
template <class T>
void godunov(const Grid& g, const T* U, T* Un, T dtdx, T ch, T decay, const Phys<T>& P, T* resid,
             const T* faces, T* work, const Drag<T>& drag, const Rad<T>& rad = Rad<T>{nullptr, 0},
             Census* census = nullptr) {
  const long nc = (long)g.nx * g.ny * g.nz;
  const bool CT = faces != nullptr;
  unsigned long long n_solves = 0, n_ref = 0, n_rel = 0;
  const long nxy = (long)g.nx * g.ny;
  const long c0 = g.zhi > g.zlo ? (long)g.zlo * nxy : 0, c1 = g.zhi > g.zlo ? (long)g.zhi * nxy : nc;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : n_solves, n_ref, n_rel)
  for (long c = c0; c < c1; ++c) {
    int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long)g.nx * g.ny));
    // census of this cell's three lower faces (each face of the grid counted once)
    Census loc{0, 0, 0};
    Census* cen = census ? &loc : nullptr;
    const bool fo = rad.corr != nullptr && (rad.flags & RAD_FIRST_ORDER) != 0;
    const bool msk = rad.corr != nullptr && (rad.flags & RAD_MASKED) != 0;
    // masked fallback: the mask of the cell at periodic offset (di, dj, dk) from this one
    auto masked_at = [&](int di, int dj, int dk) { return msk && rad.mask[per(g, i + di, j + dj, k + dk)] > T(0); };
    Edges<T> ec = mh_edges(g, U, nc, i, j, k, dtdx, P, fo || masked_at(0, 0, 0));
    Q<T> Fl[3], Fh[3];
    const int off[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int d = 0; d < 3; ++d) {
      const bool mm = masked_at(-off[d][0], -off[d][1], -off[d][2]), m0 = masked_at(0, 0, 0);
      const bool mp = masked_at(off[d][0], off[d][1], off[d][2]);
      Edges<T> em = mh_edges(g, U, nc, i - off[d][0], j - off[d][1], k - off[d][2], dtdx, P, fo || mm);
      Edges<T> ep = mh_edges(g, U, nc, i + off[d][0], j + off[d][1], k + off[d][2], dtdx, P, fo || mp);
      // face states mh + offset, drag-propagated when drag is on, plus the radiation velocity
      // correction of the owning cell (integrator_ref.jl:28-39)
      auto face = [&](const Edges<T>& e, const Q<T>& off, long cell) {
        Q<T> q = drag.on ? drag_predict_face(qadd(e.m0, off), qadd(e.mh, off), drag.qh, drag.v0) : qadd(e.mh, off);
        if (rad.corr)
          for (int v = 1; v <= 3; ++v) q[v] += rad.corr[v * nc + cell];
        return q;
      };
      const long cm = per(g, i - off[d][0], j - off[d][1], k - off[d][2]);
      const long cp = per(g, i + off[d][0], j + off[d][1], k + off[d][2]);
      Q<T> Ll = face(em, em.dR[d], cm), Rl = face(ec, ec.dL[d], c);
      Q<T> Lh = face(ec, ec.dR[d], c), Rh = face(ep, ep.dL[d], cp);
      if (CT) {
        T bl = faces[d * nc + c];
        T bh = faces[d * nc + per(g, i + off[d][0], j + off[d][1], k + off[d][2])];
        Ll[5 + d] = bl; Rl[5 + d] = bl; Lh[5 + d] = bh; Rh[5 + d] = bh;
        Fl[d] = riemann_ct(Ll, Rl, d, P, cen, mm || m0); Fh[d] = riemann_ct(Lh, Rh, d, P, nullptr, m0 || mp);
      } else {
        Fl[d] = riemann(Ll, Rl, d, ch, P, cen, mm || m0); Fh[d] = riemann(Lh, Rh, d, ch, P, nullptr, m0 || mp);
      }
    }
    Q<T> U0; for (int v = 0; v < 9; ++v) U0[v] = U[v * nc + c];
    if (CT) {
      work[W_MFX * nc + c] = Fl[0][0]; work[W_MFY * nc + c] = Fl[1][0]; work[W_MFZ * nc + c] = Fl[2][0];
      work[W_FXBY * nc + c] = Fl[0][6]; work[W_FXBZ * nc + c] = Fl[0][7];
      work[W_FYBX * nc + c] = Fl[1][5]; work[W_FYBZ * nc + c] = Fl[1][7];
      work[W_FZBX * nc + c] = Fl[2][5]; work[W_FZBY * nc + c] = Fl[2][6];
      const Q<T> qz{{T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0), T(0)}};
      Q<T> qc = drag.on ? drag_predict_face(qadd(ec.m0, qz), qadd(ec.mh, qz), drag.qh, drag.v0) : ec.mh;
      if (rad.corr)
        for (int v = 1; v <= 3; ++v) qc[v] += rad.corr[v * nc + c];
      work[W_ECX * nc + c] = qc[3] * U0[6] - qc[2] * U0[7];
      work[W_ECY * nc + c] = qc[1] * U0[7] - qc[3] * U0[5];
      work[W_ECZ * nc + c] = qc[2] * U0[5] - qc[1] * U0[6];
    }
    T dU[9];
    for (int v = 0; v < 9; ++v) dU[v] = dtdx * (((Fl[0][v] - Fh[0][v]) + (Fl[1][v] - Fh[1][v])) + (Fl[2][v] - Fh[2][v]));
    Q<T> r;
    r[0] = U0[0] + dU[0];
    if (resid) {
      // compensated: momentum (slots 0-2), E (3), B (4-6; cell B only for GLM)
      r[1] = comp_update(resid, 0 * nc + c, U0[1], dU[1]);
      r[2] = comp_update(resid, 1 * nc + c, U0[2], dU[2]);
      r[3] = comp_update(resid, 2 * nc + c, U0[3], dU[3]);
      r[4] = comp_update(resid, 3 * nc + c, U0[4], dU[4]);
      for (int b = 0; b < 3; ++b)
        r[5 + b] = CT ? U0[5 + b] + dU[5 + b] : comp_update(resid, (4 + b) * nc + c, U0[5 + b], dU[5 + b]);
    } else {
      for (int v = 1; v < 8; ++v) r[v] = U0[v] + dU[v];
    }
    r[8] = U0[8] + dU[8];
    bool bad = false;
    if (rad.corr) {
      // tracked density increment, compensated E and (GLM) cell B, admissibility flag
      // (integrator_cube.jl:85-106,412-432)
      T* cr = rad.corr;
      if (rad.flags & RAD_TRACK_DENSITY) cr[4 * nc + c] += dU[0];
      if (rad.flags & RAD_TRACK_ENERGY) r[4] = comp_update(cr, 8 * nc + c, U0[4], dU[4]);
      if ((rad.flags & RAD_TRACK_MAGNETIC) && !CT)
        for (int b = 0; b < 3; ++b) r[5 + b] = comp_update(cr, (5 + b) * nc + c, U0[5 + b], dU[5 + b]);
      if (rad.flags & RAD_CHECK) bad = inadmissible(r, P);
      // drag corrector, its work removed from E through the energy remainder when tracked
      // (drag_correct_conserved_compensated!, glm_physics.jl:374-400; _compensated_floor_update!)
      T qwork, emin;
      const T e_trial = r[4];
      r = drag_correct_parts(U0, r, drag.q, drag.v0, P.smallr, T(1e-30), qwork, emin);
      if (rad.flags & RAD_TRACK_ENERGY) {
        T e = comp_update(cr, 8 * nc + c, e_trial, -qwork);
        if (e < emin) { cr[8 * nc + c] = T(0); e = emin; }
        r[4] = e;
      } else {
        r[4] = mx(e_trial - qwork, emin);
      }
    } else if (drag.on) {
      r = drag_correct_conserved(U0, r, drag.q, drag.v0, P.smallr, T(1e-30));  // integrator_ref.jl:155-156
    }
    if (bad) r[0] = -mx(std::fabs(r[0]), mx(P.smallr, P.llf_dmin));
    for (int v = 0; v < 8; ++v) Un[v * nc + c] = r[v];
    Un[8 * nc + c] = CT ? T(0) : r[8] * decay;
    n_solves += loc.solves;
    n_ref += loc.ref_sides;
    n_rel += loc.rel_sides;
  }
  if (census) {
    census->solves += n_solves;
    census->ref_sides += n_ref;
    census->rel_sides += n_rel;
  }
}

// ct.jl:57-66
template <class T> T gs05(T Ea0, T Eam, T Eb0, T Ebm, T mA0, T mAm, T mB0, T mBm, T Er00, T Erm0, T Er0m, T Ermm) {
  const T h = T(0.5);
  auto up = [h](T m, T lower, T upper) { return m > T(0) ? lower : (m < T(0) ? upper : h * (lower + upper)); };
  T A1 = up(mA0, Erm0 - Ebm, Er00 - Eb0);
  T A3 = up(mAm, Ebm - Ermm, Eb0 - Er0m);
  T B1 = up(mB0, Er0m - Eam, Er00 - Ea0);
  T B3 = up(mBm, Eam - Ermm, Ea0 - Erm0);
  return T(0.25) * ((Ea0 + Eam + Eb0 + Ebm) + (A3 - A1) + (B3 - B1));
}

// ct.jl:71-143 — edge EMFs, face curl update (plain / compensated), cell B = face average.
template <class T> void ct_update(const Grid& g, T* Un, T* faces, T* work, T* face_resid, T dtdx) {
  const long nc = (long)g.nx * g.ny * g.nz;
  const T* W = work;
  T* ex = work + W_EX * nc; T* ey = work + W_EY * nc; T* ez = work + W_EZ * nc;
#pragma omp parallel for
  for (long c = 0; c < nc; ++c) {
    int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long)g.nx * g.ny));
    long cim = per(g, i - 1, j, k), cjm = per(g, i, j - 1, k), ckm = per(g, i, j, k - 1);
    long cimjm = per(g, i - 1, j - 1, k), cjmkm = per(g, i, j - 1, k - 1), ckmim = per(g, i - 1, j, k - 1);
    auto w = [&](int s, long x) { return W[s * nc + x]; };
    ez[c] = gs05(-w(W_FXBY, c), -w(W_FXBY, cjm), w(W_FYBX, c), w(W_FYBX, cim), w(W_MFX, c), w(W_MFX, cjm),
                 w(W_MFY, c), w(W_MFY, cim), w(W_ECZ, c), w(W_ECZ, cim), w(W_ECZ, cjm), w(W_ECZ, cimjm));
    ex[c] = gs05(-w(W_FYBZ, c), -w(W_FYBZ, ckm), w(W_FZBY, c), w(W_FZBY, cjm), w(W_MFY, c), w(W_MFY, ckm),
                 w(W_MFZ, c), w(W_MFZ, cjm), w(W_ECX, c), w(W_ECX, cjm), w(W_ECX, ckm), w(W_ECX, cjmkm));
    ey[c] = gs05(-w(W_FZBX, c), -w(W_FZBX, cim), w(W_FXBZ, c), w(W_FXBZ, ckm), w(W_MFZ, c), w(W_MFZ, cim),
                 w(W_MFX, c), w(W_MFX, ckm), w(W_ECY, c), w(W_ECY, ckm), w(W_ECY, cim), w(W_ECY, ckmim));
  }
  T* bxf = faces; T* byf = faces + nc; T* bzf = faces + 2 * nc;
#pragma omp parallel for
  for (long c = 0; c < nc; ++c) {
    int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long)g.nx * g.ny));
    long ip = per(g, i + 1, j, k), jp = per(g, i, j + 1, k), kp = per(g, i, j, k + 1);
    T dbx = dtdx * ((ez[jp] - ez[c]) - (ey[kp] - ey[c]));
    T dby = dtdx * ((ex[kp] - ex[c]) - (ez[ip] - ez[c]));
    T dbz = dtdx * ((ey[ip] - ey[c]) - (ex[jp] - ex[c]));
    if (face_resid) {
      bxf[c] = comp_update(face_resid, c, bxf[c], -dbx);
      byf[c] = comp_update(face_resid, nc + c, byf[c], -dby);
      bzf[c] = comp_update(face_resid, 2 * nc + c, bzf[c], -dbz);
    } else {
      bxf[c] -= dbx; byf[c] -= dby; bzf[c] -= dbz;
    }
  }
#pragma omp parallel for
  for (long c = 0; c < nc; ++c) {
    int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long)g.nx * g.ny));
    Un[5 * nc + c] = T(0.5) * (bxf[c] + bxf[per(g, i + 1, j, k)]);
    Un[6 * nc + c] = T(0.5) * (byf[c] + byf[per(g, i, j + 1, k)]);
    Un[7 * nc + c] = T(0.5) * (bzf[c] + bzf[per(g, i, j, k + 1)]);
  }
}

// timestep.jl:4-14
template <class T> T max_wavespeed(const Grid& g, const T* U, const Phys<T>& P) {
  const long nc = (long)g.nx * g.ny * g.nz;
  T best = T(0);
#pragma omp parallel for reduction(max : best)
  for (long c = 0; c < nc; ++c) {
    Q<T> u; for (int v = 0; v < 9; ++v) u[v] = U[v * nc + c];
    Q<T> q = cons2prim(u, P.gamma, P.smallr, P.pfl);
    T sx = std::fabs(q[1]) + fast_speed(q, P.gamma, q[5]);
    T sy = std::fabs(q[2]) + fast_speed(q, P.gamma, q[6]);
    T sz = std::fabs(q[3]) + fast_speed(q, P.gamma, q[7]);
    T s = mx(sx, mx(sy, sz));
    best = mx(best, s);
  }
  return best;
}

// diagnostics.jl:6-20 — max |div B| by BC-aware centred differences
template <class T> T max_divb(const Grid& g, const T* U, T dx) {
  const long nc = (long)g.nx * g.ny * g.nz;
  const T* bx = U + 5 * nc; const T* by = U + 6 * nc; const T* bz = U + 7 * nc;
  T inv2dx = T(1) / (T(2) * dx);
  T best = T(0);
#pragma omp parallel for reduction(max : best)
  for (long c = 0; c < nc; ++c) {
    int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long)g.nx * g.ny));
    int ip, fxp, im, fxm, jp, fyp, jm, fym, kp, fzp, km, fzm;
    bcidx(i + 1, g.nx, g.bc[0], ip, fxp); bcidx(i - 1, g.nx, g.bc[0], im, fxm);
    bcidx(j + 1, g.ny, g.bc[1], jp, fyp); bcidx(j - 1, g.ny, g.bc[1], jm, fym);
    bcidx(k + 1, g.nz, g.bc[2], kp, fzp); bcidx(k - 1, g.nz, g.bc[2], km, fzm);
    T db = (bx[lin(g, ip, j, k)] * T(fxp) - bx[lin(g, im, j, k)] * T(fxm) + by[lin(g, i, jp, k)] * T(fyp) -
            by[lin(g, i, jm, k)] * T(fym) + bz[lin(g, i, j, kp)] * T(fzp) - bz[lin(g, i, j, km)] * T(fzm)) * inv2dx;
    best = mx(best, std::fabs(db));
  }
  return best;
}

// ct.jl:176-185
template <class T> T max_divb_face(const Grid& g, const T* faces, T dx) {
  const long nc = (long)g.nx * g.ny * g.nz;
  const T* bxf = faces; const T* byf = faces + nc; const T* bzf = faces + 2 * nc;
  T invdx = T(1) / dx; T best = T(0);
#pragma omp parallel for reduction(max : best)
  for (long c = 0; c < nc; ++c) {
    int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long)g.nx * g.ny));
    T d = std::fabs(((bxf[per(g, i + 1, j, k)] - bxf[c]) + (byf[per(g, i, j + 1, k)] - byf[c]) +
                     (bzf[per(g, i, j, k + 1)] - bzf[c])) * invdx);
    best = mx(best, d);
  }
  return best;
}

// ct.jl:310-320 (edge potential -> faces) and :205-219 (cell B from faces, E keeps p)
template <class T> void ct_faces_from_potential(const Grid& g, const T* A, T* faces, T* U, T dx) {
  const long nc = (long)g.nx * g.ny * g.nz;
  const T* Ax = A; const T* Ay = A + nc; const T* Az = A + 2 * nc;
  T invdx = T(1) / dx;
  for (long c = 0; c < nc; ++c) {
    int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long)g.nx * g.ny));
    faces[c] = ((Az[per(g, i, j + 1, k)] - Az[c]) - (Ay[per(g, i, j, k + 1)] - Ay[c])) * invdx;
    faces[nc + c] = ((Ax[per(g, i, j, k + 1)] - Ax[c]) - (Az[per(g, i + 1, j, k)] - Az[c])) * invdx;
    faces[2 * nc + c] = ((Ay[per(g, i + 1, j, k)] - Ay[c]) - (Ax[per(g, i, j + 1, k)] - Ax[c])) * invdx;
  }
  for (long c = 0; c < nc; ++c) {
    int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((long)g.nx * g.ny));
    T bx = T(0.5) * (faces[c] + faces[per(g, i + 1, j, k)]);
    T by = T(0.5) * (faces[nc + c] + faces[nc + per(g, i, j + 1, k)]);
    T bz = T(0.5) * (faces[2 * nc + c] + faces[2 * nc + per(g, i, j, k + 1)]);
    T ox = U[5 * nc + c], oy = U[6 * nc + c], oz = U[7 * nc + c];
    U[4 * nc + c] += T(0.5) * ((bx * bx + by * by + bz * bz) - (ox * ox + oy * oy + oz * oz));
    U[5 * nc + c] = bx; U[6 * nc + c] = by; U[7 * nc + c] = bz; U[8 * nc + c] = T(0);
  }
}

template <class T> void totals(const Grid& g, const T* U, double out[8]) {
  const long nc = (long)g.nx * g.ny * g.nz;
  const int map[8] = {0, 1, 2, 3, 4, 5, 6, 7};
  for (int q = 0; q < 8; ++q) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s)
    for (long c = 0; c < nc; ++c) s += (double)U[map[q] * nc + c];
    out[q] = s;
  }
}

}  // namespace

extern "C" {

// Parameter block shared with the Python wrapper (oracle.py).
struct oracle_params {
  int nx, ny, nz;
  int bc[3];
  int recon, riemann;
  double gamma, smallr, pfl, llf_dmin, llf_pmin;
  double hlld_dtol_rel;  // 0: the reference's HLLD degeneracy test; 1e-5: the relative test
  int zlo, zhi;          // planes a Godunov step updates (zhi <= zlo: all)
};

#define ORACLE_DEFS(T, SUF)                                                                               \
  static Phys<T> phys_##SUF(const oracle_params* p) {                                                     \
    return Phys<T>{T(p->gamma), T(p->smallr), T(p->pfl), T(p->llf_dmin), T(p->llf_pmin), p->recon, p->riemann, \
                   T(p->hlld_dtol_rel)};                                                                   \
  }                                                                                                        \
  static Grid grid_##SUF(const oracle_params* p) {                                                      \
    return Grid{p->nx, p->ny, p->nz, {p->bc[0], p->bc[1], p->bc[2]}, p->zlo, p->zhi};                     \
  }                                                                                                        \
  static Drag<T> no_drag_##SUF() { return Drag<T>{false, T(0), T(0), {T(0), T(0), T(0)}}; }                 \
  static Drag<T> drag_##SUF(double q, const double* v0) {                                                  \
    Drag<T> d{true, T(0.5) * T(q), T(q), {T(0), T(0), T(0)}};                                            \
    if (v0) for (int c = 0; c < 3; ++c) d.v0[c] = T(v0[c]);                                               \
    return d;                                                                                              \
  }                                                                                                        \
  void oracle_step_glm_##SUF(const oracle_params* p, const T* U, T* Un, double dtdx, double ch, double decay, T* resid) { \
    godunov<T>(grid_##SUF(p), U, Un, T(dtdx), T(ch), T(decay), phys_##SUF(p), resid, nullptr, nullptr,    \
               no_drag_##SUF());                                                                  \
  }                                                                                                        \
  void oracle_step_glm_census_##SUF(const oracle_params* p, const T* U, T* Un, double dtdx, double ch, double decay, \
                                    unsigned long long* out) {                                             \
    Census cs{0, 0, 0};                                                                                    \
    godunov<T>(grid_##SUF(p), U, Un, T(dtdx), T(ch), T(decay), phys_##SUF(p), nullptr, nullptr, nullptr,  \
               no_drag_##SUF(), Rad<T>{nullptr, 0}, &cs);                                                  \
    out[0] = cs.solves; out[1] = cs.ref_sides; out[2] = cs.rel_sides;                                      \
  }                                                                                                        \
  void oracle_step_glm_drag_##SUF(const oracle_params* p, const T* U, T* Un, double dtdx, double ch, double decay, \
                                  double q, const double* v0) {                                           \
    godunov<T>(grid_##SUF(p), U, Un, T(dtdx), T(ch), T(decay), phys_##SUF(p), nullptr, nullptr, nullptr,  \
               drag_##SUF(q, v0));                                                                         \
  }                                                                                                        \
  void oracle_step_ct_##SUF(const oracle_params* p, const T* U, T* Un, T* faces, T* work, double dtdx,      \
                            T* resid, T* face_resid) {                                                    \
    Grid g = grid_##SUF(p);                                                                               \
    godunov<T>(g, U, Un, T(dtdx), T(0), T(1), phys_##SUF(p), resid, faces, work, no_drag_##SUF()); \
    ct_update<T>(g, Un, faces, work, face_resid, T(dtdx));                                                \
  }                                                                                                        \
  void oracle_step_glm_rad_##SUF(const oracle_params* p, const T* U, T* Un, double dtdx, double ch, double decay,  \
                                 double q, T* corr, int flags) {                                          \
    Grid g = grid_##SUF(p);                                                                               \
    const long nc = (long)g.nx * g.ny * g.nz;                                                             \
    std::vector<T> mask((flags & RAD_MASKED) ? corr + 4 * nc : corr,                                       \
                        (flags & RAD_MASKED) ? corr + 5 * nc : corr);                                      \
    godunov<T>(g, U, Un, T(dtdx), T(ch), T(decay), phys_##SUF(p), nullptr, nullptr, nullptr,              \
               drag_##SUF(q, nullptr), Rad<T>{corr, flags, mask.data()});                                  \
  }                                                                                                        \
  void oracle_step_ct_rad_##SUF(const oracle_params* p, const T* U, T* Un, T* faces, T* work, T* face_resid, \
                                double dtdx, double q, T* corr, int flags) {                              \
    Grid g = grid_##SUF(p);                                                                               \
    godunov<T>(g, U, Un, T(dtdx), T(0), T(1), phys_##SUF(p), nullptr, faces, work, drag_##SUF(q, nullptr), \
               Rad<T>{corr, flags});                                                                       \
    ct_update<T>(g, Un, faces, work, (flags & RAD_TRACK_MAGNETIC) ? face_resid : nullptr, T(dtdx));       \
  }                                                                                                        \
  void oracle_step_ct_drag_##SUF(const oracle_params* p, const T* U, T* Un, T* faces, T* work, double dtdx, \
                                 double q, const double* v0) {                                            \
    Grid g = grid_##SUF(p);                                                                               \
    godunov<T>(g, U, Un, T(dtdx), T(0), T(1), phys_##SUF(p), nullptr, faces, work, drag_##SUF(q, v0));    \
    ct_update<T>(g, Un, faces, work, nullptr, T(dtdx));                                                   \
  }                                                                                                        \
  double oracle_max_wavespeed_##SUF(const oracle_params* p, const T* U) {                                 \
    return (double)max_wavespeed<T>(grid_##SUF(p), U, phys_##SUF(p));                                     \
  }                                                                                                        \
  double oracle_max_divb_##SUF(const oracle_params* p, const T* U, double dx) {                           \
    return (double)max_divb<T>(grid_##SUF(p), U, T(dx));                                                  \
  }                                                                                                        \
  double oracle_max_divb_face_##SUF(const oracle_params* p, const T* faces, double dx) {                  \
    return (double)max_divb_face<T>(grid_##SUF(p), faces, T(dx));                                         \
  }                                                                                                        \
  void oracle_ct_faces_from_potential_##SUF(const oracle_params* p, const T* A, T* faces, T* U, double dx) { \
    ct_faces_from_potential<T>(grid_##SUF(p), A, faces, U, T(dx));                                        \
  }                                                                                                        \
  void oracle_totals_##SUF(const oracle_params* p, const T* U, double* out) { totals<T>(grid_##SUF(p), U, out); }

ORACLE_DEFS(float, f32)
ORACLE_DEFS(double, f64)

}  // extern "C"
