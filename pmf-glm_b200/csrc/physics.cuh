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
// RS_HLLD_CENSUS: HLLD that also counts its single-star degeneracy cases (HlldCensus); only the
// census step instantiates it.
enum { RS_HLLD = 0, RS_HLL = 1, RS_LLF = 2, RS_HLLD_CENSUS = 3 };
enum { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECT = 2 };

struct F9 {
  float v[9];
  __device__ __forceinline__ float& operator[](int i) { return v[i]; }
  __device__ __forceinline__ const float& operator[](int i) const { return v[i]; }
};

struct Phys {
  float gamma, smallr, pfl, llf_dmin, llf_pmin;
  // HLLD single-star degeneracy test |denK| < max(1e-12, dtol_rel * bn^2); 0 is the reference's
  // absolute test |denK| < 1e-12 (glm_physics.jl:257)
  float dtol_rel;
};

// Per-thread counts of the HLLD degeneracy census (RS_HLLD_CENSUS): solves, single-star sides
// with |denK| < 1e-12 (the reference's degenerate branch) and sides with 1e-12 <= |denK| <
// 1e-5 bn^2 (sent to the degenerate branch by the relative test only).
struct HlldCensus {
  unsigned solves, ref_sides, rel_sides;
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

// ---- packed FP32 pairs (sm_100 FFMA2 / FMUL2 / FADD2): two independent evaluations of the
// same expression in one instruction, each lane rounded exactly as the scalar operation ----
__device__ __forceinline__ float2 p2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 pb(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a*b - c*d per lane
__device__ __forceinline__ float2 msub2(float2 a, float2 b, float2 c, float2 d) {
  return fma2(a, b, make_float2(-(c.x * d.x), -(c.y * d.y)));
}
struct P9 {
  float2 v[9];
  __device__ __forceinline__ float2& operator[](int i) { return v[i]; }
  __device__ __forceinline__ const float2& operator[](int i) const { return v[i]; }
};

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

// minmod limiter (glm_physics.jl:54-59); MonCen is half_moncen below
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

// Offsets kept or replaced by exact zeros (keep = false: the piecewise-constant states of a
// first-order fallback). A select, not a product: an Inf or NaN offset of a bad state still
// gives a zero offset, as the reference's assignment of zeros does (integrator_cube.jl:168-171).
template <int RECON> __device__ __forceinline__ void keep_offsets(Offsets<RECON>& o, bool keep) {
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    o.dR[i] = keep ? o.dR[i] : 0.0f;
    if constexpr (RECON == RECON_PPM) o.dL[i] = keep ? o.dL[i] : 0.0f;
  }
}

// min(|a|, |b|) carrying the sign sign(a) XOR sign(b) (PTX min.xorsign.abs, one instruction).
__device__ __forceinline__ float min_xorsign_abs(float a, float b) {
  float r;
  asm("min.xorsign.abs.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
// Half the MonCen slope, 0.5*moncen(dl, dr) of glm_physics.jl:47-53, from dl, dr and
// q = (dl+dr)/4. With the scalings by powers of two folded, the reference's value is
// 0.5*sgn*min(2*min|dl|,|dr|, |(dl+dr)/2|) = sgn(q)*min(min(|dl|,|dr|), |q|) when dl*dr > 0 and
// 0 otherwise. t = min.xorsign.abs(dl, dr) has magnitude min(|dl|,|dr|) and is positive exactly
// when dl and dr have the same sign, so max(t, 0) is zero wherever the reference returns zero,
// and min.xorsign.abs(max(t, 0), q) carries sgn(q): three instructions, the same value (up to
// the sign of a zero result), every step exact.
__device__ __forceinline__ float half_moncen(float dl, float dr, float q) {
  return min_xorsign_abs(fmaxf(min_xorsign_abs(dl, dr), 0.0f), q);
}
// Two fields at once: the differences and the quarter sum as packed pairs (each lane rounded as
// the scalar operation), the limiter per lane.
__device__ __forceinline__ float2 half_moncen2(float2 mm, float2 m0, float2 mp) {
  const float2 dl = sub2(m0, mm), dr = sub2(mp, m0);
  const float2 q = mul2(pb(0.25f), add2(dl, dr));
  return make_float2(half_moncen(dl.x, dr.x, q.x), half_moncen(dl.y, dr.y, q.y));
}

template <int RECON>
__device__ __forceinline__ Offsets<RECON> recon(const F9& mm, const F9& m0, const F9& mp) {
  Offsets<RECON> o;
  if constexpr (RECON == RECON_PLM) {
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
      const float2 h = half_moncen2(p2(mm[i], mm[i + 1]), p2(m0[i], m0[i + 1]), p2(mp[i], mp[i + 1]));
      o.dR[i] = h.x;
      o.dR[i + 1] = h.y;
    }
    const float dl = m0[8] - mm[8], dr = mp[8] - m0[8];
    o.dR[8] = half_moncen(dl, dr, 0.25f * (dl + dr));
  } else if constexpr (RECON == RECON_PLM_MINMOD) {
#pragma unroll
    for (int i = 0; i < 9; ++i) o.dR[i] = 0.5f * minmod(m0[i] - mm[i], mp[i] - m0[i]);
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i) {
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

// x-normal flux of two primitive states at once (lane x and lane y), glm_physics.jl:28-34.
__device__ __forceinline__ P9 phys_flux_x2(const P9& q, float g) {
  const float2 rho = q[0], vx = q[1], vy = q[2], vz = q[3], p = q[4], bx = q[5], by = q[6], bz = q[7];
  const float2 b2 = fma2(bz, bz, fma2(by, by, mul2(bx, bx)));
  const float2 half = pb(0.5f);
  const float2 ptot = fma2(half, b2, p);
  const float2 v2 = fma2(vz, vz, fma2(vy, vy, mul2(vx, vx)));
  const float ig = 1.0f / (g - 1.0f);
  const float2 E = fma2(half, b2, fma2(mul2(half, rho), v2, mul2(p, pb(ig))));
  const float2 vb = fma2(vz, bz, fma2(vy, by, mul2(vx, bx)));
  const float2 m = mul2(rho, vx);
  P9 f;
  f[0] = m;
  f[1] = sub2(fma2(m, vx, ptot), mul2(bx, bx));
  f[2] = sub2(mul2(m, vy), mul2(bx, by));
  f[3] = sub2(mul2(m, vz), mul2(bx, bz));
  f[4] = sub2(mul2(add2(E, ptot), vx), mul2(bx, vb));
  f[5] = pb(0.0f);
  f[6] = sub2(mul2(vx, by), mul2(vy, bx));
  f[7] = sub2(mul2(vx, bz), mul2(vz, bx));
  f[8] = pb(0.0f);
  return f;
}

// flux difference F(m0 + dR) - F(m0 + dL) along axis D (one term of the Hancock predictor,
// glm_physics.jl:225-231); the flux of the two face states is evaluated as one packed pair (the
// states themselves are formed by scalar adds, which write the pair's registers directly)
template <int D, int RECON>
__device__ __forceinline__ F9 hancock_term(const F9& m0, const Offsets<RECON>& o, float g) {
  // global -> D-normal component order, as rot_to<D>
  constexpr int perm[3][9] = {{0, 1, 2, 3, 4, 5, 6, 7, 8}, {0, 2, 3, 1, 4, 6, 7, 5, 8}, {0, 3, 1, 2, 4, 7, 5, 6, 8}};
  P9 q;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int j = perm[D][i];
    q[i] = make_float2(m0[j] + o.dR[j], m0[j] + o.l(j));
  }
  const P9 f = phys_flux_x2(q, g);
  F9 d;
  // back to the global order (rot_back<D>) while taking the difference of the two lanes
#pragma unroll
  for (int i = 0; i < 9; ++i) d[perm[D][i]] = f[i].x - f[i].y;
  return d;
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
// HLLD, Miyoshi & Kusano 2005 (glm_physics.jl:255-307). The left and right halves of the
// solver are the same algebra on the two states, so they run as packed pairs (lane x = L,
// lane y = R); the scalar parts are the wave speeds, the contact speed and the doubly-starred
// state, which mix both sides.
__device__ __forceinline__ F9 hlld_x(const F9& L, const F9& R, float g, float bn, float fbn, float fpsi,
                                     float dtol_rel, HlldCensus* cen = nullptr) {
  const float2 d = p2(L[0], R[0]), u = p2(L[1], R[1]), v = p2(L[2], R[2]), w = p2(L[3], R[3]);
  const float2 p = p2(L[4], R[4]), by = p2(L[6], R[6]), bz = p2(L[7], R[7]);
  const float2 half = pb(0.5f);
  const float bn2 = bn * bn;
  const float2 b2 = fma2(bz, bz, fma2(by, by, pb(bn2)));
  const float2 pt = fma2(half, b2, p);
  const float ig = 1.0f / (g - 1.0f);
  const float2 E = fma2(half, b2, fma2(mul2(half, d), fma2(w, w, fma2(v, v, mul2(u, u))), mul2(p, pb(ig))));
  // fast speeds (glm_physics.jl:24-27) with the normal field bn
  const float2 id = p2(1.0f / L[0], 1.0f / R[0]);
  const float2 c2 = mul2(mul2(pb(g), p), id);
  const float2 bb = mul2(b2, id);
  const float2 d2 = mul2(half, add2(bb, c2));
  const float2 disc = sub2(mul2(d2, d2), mul2(mul2(c2, pb(bn2)), id));
  const float2 in = add2(d2, p2(sqrtf(fmaxf(disc.x, 0.0f)), sqrtf(fmaxf(disc.y, 0.0f))));
  const float cfL = sqrtf(in.x), cfR = sqrtf(in.y);
  const float cf = fmaxf(cfL, cfR);
  const float SL = fminf(fminf(u.x, u.y) - cf, 0.0f);
  const float SR = fmaxf(fmaxf(u.x, u.y) + cf, 0.0f);
  const float2 S = p2(SL, SR);
  const float2 Su = sub2(S, u);         // S - u per side
  const float2 dSu = mul2(Su, d);       // d (S - u)
  const float den = dSu.y - dSu.x;
  const float2 dSuu = mul2(dSu, u);
  const float SM = ((dSuu.y - dSuu.x) - pt.y + pt.x) / den;
  const float pts = ((dSu.y * pt.x - dSu.x * pt.y) + d.x * d.y * Su.y * Su.x * (u.y - u.x)) / den;
  const float2 SSM = sub2(S, pb(SM));   // S - SM per side
  const float2 ds = mul2(dSu, p2(1.0f / SSM.x, 1.0f / SSM.y));
  const float dLs = fmaxf(ds.x, 1e-12f), dRs = fmaxf(ds.y, 1e-12f);
  const float2 dst = p2(dLs, dRs);
  const float sqL = sqrtf(dLs), sqR = sqrtf(dRs);
  const float abn = fabsf(bn);
  const float SLs = SM - abn / sqL, SRs = SM + abn / sqR;
  // single-starred transverse states of both sides (glm_physics.jl:255-263)
  const float2 denK = fma2(dSu, SSM, pb(-bn2));
  const float2 nK = fma2(dSu, Su, pb(-bn2));       // d (S - u)^2 - bn^2
  const float2 iK = p2(1.0f / denK.x, 1.0f / denK.y);
  const float2 fac = mul2(mul2(pb(bn), sub2(pb(SM), u)), iK);
  const float2 rK = mul2(nK, iK);
  // Degenerate star state (the fast and Alfven speeds coincide). The reference tests
  // |denK| < 1e-12 (dtol_rel = 0), which is below the FP32 rounding of denK = d(S-u)(S-SM) - bn^2
  // (a difference of two terms of size bn^2): a 1-ulp residue then makes the single-star states
  // ~1/denK and the fan flux depends on a cancellation (S*_L - S_L) * U*_L. The relative mode
  // (dtol_rel = 1e-5) sends faces with |denK| within 1e-5 bn^2 of zero to the degenerate branch.
  const float dtol = fmaxf(1e-12f, dtol_rel * bn2);
  const bool degL = fabsf(denK.x) < dtol, degR = fabsf(denK.y) < dtol;
  if (cen != nullptr) {
    const float t5 = 1e-5f * bn2, aL = fabsf(denK.x), aR = fabsf(denK.y);
    cen->solves += 1;
    cen->ref_sides += (aL < 1e-12f ? 1u : 0u) + (aR < 1e-12f ? 1u : 0u);
    cen->rel_sides += (aL >= 1e-12f && aL < t5 ? 1u : 0u) + (aR >= 1e-12f && aR < t5 ? 1u : 0u);
  }
  float2 vs = sub2(v, mul2(by, fac)), ws = sub2(w, mul2(bz, fac));
  float2 bys = mul2(by, rK), bzs = mul2(bz, rK);
  if (degL) { vs.x = v.x; ws.x = w.x; bys.x = by.x; bzs.x = bz.x; }
  if (degR) { vs.y = v.y; ws.y = w.y; bys.y = by.y; bzs.y = bz.y; }
  const float2 vdb = fma2(w, bz, fma2(v, by, mul2(u, pb(bn))));
  const float2 vdbs = fma2(ws, bzs, fma2(vs, bys, pb(SM * bn)));
  // E* = ((S - u) E - pt u + pts SM + bn (v.b - v*.b*)) / (S - SM)
  const float2 Enum = fma2(pb(bn), sub2(vdb, vdbs), add2(sub2(mul2(Su, E), mul2(pt, u)), pb(pts * SM)));
  const float2 Es = mul2(Enum, p2(1.0f / SSM.x, 1.0f / SSM.y));
  const float sgn = bn >= 0.0f ? 1.0f : -1.0f;
  const float invsum = 1.0f / (sqL + sqR);
  const float vyss = (sqL * vs.x + sqR * vs.y + (bys.y - bys.x) * sgn) * invsum;
  const float vzss = (sqL * ws.x + sqR * ws.y + (bzs.y - bzs.x) * sgn) * invsum;
  const float byss = (sqL * bys.y + sqR * bys.x + sqL * sqR * (vs.y - vs.x) * sgn) * invsum;
  const float bzss = (sqL * bzs.y + sqR * bzs.x + sqL * sqR * (ws.y - ws.x) * sgn) * invsum;
  const float vdbss = SM * bn + vyss * byss + vzss * bzss;
  // E** = E* -+ sqrt(d*) (v*.b* - v**.b**) sgn
  const float2 Ess = fma2(mul2(p2(-sqL, sqR), pb(sgn)), sub2(vdbs, pb(vdbss)), Es);
  // only the selected fan state is assembled: the four branches of glm_physics.jl:297-305
  F9 f;
  const bool left = SM >= 0.0f;
  const float dK = left ? d.x : d.y, uK = left ? u.x : u.y, vK = left ? v.x : v.y, wK = left ? w.x : w.y;
  const float pK = left ? p.x : p.y, byK = left ? by.x : by.y, bzK = left ? bz.x : bz.y;
  const float EK = left ? E.x : E.y, SK = left ? SL : SR, dKs = left ? dLs : dRs;
  const float vKs = left ? vs.x : vs.y, wKs = left ? ws.x : ws.y, byKs = left ? bys.x : bys.y;
  const float bzKs = left ? bzs.x : bzs.y, EKs = left ? Es.x : Es.y, EKss = left ? Ess.x : Ess.y;
  const float SKs = left ? SLs : SRs;
  const bool outer = left ? (SLs >= 0.0f) : (SRs < 0.0f);
  const F9 FK = phys_flux_x(F9{{dK, uK, vK, wK, pK, bn, byK, bzK, 0.0f}}, g);
  const float UK[8] = {dK, dK * uK, dK * vK, dK * wK, EK, bn, byK, bzK};
  const float UKs[8] = {dKs, dKs * SM, dKs * vKs, dKs * wKs, EKs, bn, byKs, bzKs};
  if (outer) {
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FK[i] + SK * (UKs[i] - UK[i]);
  } else {
    const float UKss[8] = {dKs, dKs * SM, dKs * vyss, dKs * vzss, EKss, bn, byss, bzss};
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = FK[i] + SKs * UKss[i] - (SKs - SK) * UKs[i] - SK * UK[i];
  }
  f[5] = fbn;
  f[8] = fpsi;
  return f;
}

// GLM Riemann problem on a D-normal face (glm_physics.jl:317-329): floors, Dedner pair,
// the selected solver (HLLD with the LLF fallback at low density/pressure), rotate back.
// ich = 1/ch, formed once per launch: the cleaned normal field every solve starts from then
// waits on a multiply, not on a division.
// force_llf: LLF on this face whatever the solver (the masked fallback of the cube kernel,
// integrator_cube.jl:68-83); false except in the radiation-coupled step.
template <int D, int RSOL>
__device__ __forceinline__ F9 riemann_glm(const F9& Lq, const F9& Rq, float ch, float ich, const Phys& P,
                                          HlldCensus* cen = nullptr, bool force_llf = false) {
  F9 L = rot_to<D>(Lq), R = rot_to<D>(Rq);
  L[0] = fmaxf(L[0], P.smallr); L[4] = fmaxf(L[4], P.pfl);
  R[0] = fmaxf(R[0], P.smallr); R[4] = fmaxf(R[4], P.pfl);
  float bns = 0.5f * (L[5] + R[5]) - 0.5f * (R[8] - L[8]) * ich;
  float psis = 0.5f * (L[8] + R[8]) - 0.5f * ch * (R[5] - L[5]);
  float fbn = psis, fpsi = ch * ch * bns;
  L[5] = bns; R[5] = bns;
  F9 f;
  if constexpr (RSOL == RS_LLF) {
    f = llf_x(L, R, P.gamma, ch, fbn, fpsi);
  } else if constexpr (RSOL == RS_HLL) {
    if (force_llf) f = llf_x(L, R, P.gamma, ch, fbn, fpsi);
    else f = hll_x(L, R, P.gamma, bns, fbn, fpsi);
  } else {
    bool uself = force_llf || (P.llf_dmin > 0.0f && fminf(L[0], R[0]) < P.llf_dmin) ||
                 (P.llf_pmin > 0.0f && fminf(L[4], R[4]) < P.llf_pmin);
    if (uself) f = llf_x(L, R, P.gamma, ch, fbn, fpsi);
    else f = hlld_x(L, R, P.gamma, bns, fbn, fpsi, P.dtol_rel, cen);
  }
  return rot_back<D>(f);
}

// Constrained-transport Riemann problem (glm_physics.jl:336-348): the caller has put the
// staggered face value into both states' normal-B slot; no psi, ch = 0 in the LLF speed.
template <int D, int RSOL>
__device__ __forceinline__ F9 riemann_ct(const F9& Lq, const F9& Rq, const Phys& P, HlldCensus* cen = nullptr,
                                         bool force_llf = false) {
  F9 L = rot_to<D>(Lq), R = rot_to<D>(Rq);
  L[0] = fmaxf(L[0], P.smallr); L[4] = fmaxf(L[4], P.pfl); L[8] = 0.0f;
  R[0] = fmaxf(R[0], P.smallr); R[4] = fmaxf(R[4], P.pfl); R[5] = L[5]; R[8] = 0.0f;
  float bns = L[5];
  F9 f;
  if constexpr (RSOL == RS_LLF) {
    f = llf_x(L, R, P.gamma, 0.0f, 0.0f, 0.0f);
  } else if constexpr (RSOL == RS_HLL) {
    if (force_llf) f = llf_x(L, R, P.gamma, 0.0f, 0.0f, 0.0f);
    else f = hll_x(L, R, P.gamma, bns, 0.0f, 0.0f);
  } else {
    bool uself = force_llf || (P.llf_dmin > 0.0f && fminf(L[0], R[0]) < P.llf_dmin) ||
                 (P.llf_pmin > 0.0f && fminf(L[4], R[4]) < P.llf_pmin);
    if (uself) f = llf_x(L, R, P.gamma, 0.0f, 0.0f, 0.0f);
    else f = hlld_x(L, R, P.gamma, bns, 0.0f, 0.0f, P.dtol_rel, cen);
  }
  return rot_back<D>(f);
}

// `cen` is read only by the census instantiation (RS_HLLD_CENSUS); pass it for the faces to be
// counted, nullptr otherwise.
template <int D, int RSOL, bool CT>
__device__ __forceinline__ F9 riemann(const F9& L, const F9& R, float ch, float ich, const Phys& P,
                                      HlldCensus* cen = nullptr, bool force_llf = false) {
  if constexpr (RSOL != RS_HLLD_CENSUS) cen = nullptr;
  if constexpr (CT) return riemann_ct<D, RSOL>(L, R, P, cen, force_llf);
  else return riemann_glm<D, RSOL>(L, R, ch, ich, P, cen, force_llf);
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

// ---- linear (Compton) drag toward a target velocity, glm_physics.jl:63-172 ------------------
// Coefficients of one step with impulse q = Gamma*dt (computed on the host in FP32 with the
// reference's formulas): the face prediction uses the half-step pair (exp(-q/2), phi1(q/2)),
// the cell corrector the full-step pair and the integrated-work coefficients A, C, D.
struct DragCoef {
  float v0[3];       // target velocity
  float fdecay, fphi1;
  float decay, phi1, A, C, D;
};

// Drag-propagated Hancock prediction (glm_physics.jl:71-84 with the face offset folded):
// the face velocity v0 + fd*((m0+d) - v0) + fp*((mh+d) - (m0+d)) equals mh' + fd*d with
// mh' = v0 + fd*(m0 - v0) + fp*(mh - m0), so the cell's predicted velocity is replaced by mh'
// and its velocity offsets are scaled by fd. Density, pressure, B and psi keep their
// hyperbolic midpoint values.
template <int RECON>
__device__ __forceinline__ void drag_predict_cell(F9& mh, const F9& m0, Offsets<RECON>& ox, Offsets<RECON>& oy,
                                                  Offsets<RECON>& oz, const DragCoef& k) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float v0 = k.v0[c];
    mh[1 + c] = v0 + k.fdecay * (m0[1 + c] - v0) + k.fphi1 * (mh[1 + c] - m0[1 + c]);
    ox.dR[1 + c] *= k.fdecay;
    oy.dR[1 + c] *= k.fdecay;
    oz.dR[1 + c] *= k.fdecay;
    if constexpr (RECON == RECON_PPM) {
      ox.dL[1 + c] *= k.fdecay;
      oy.dL[1 + c] *= k.fdecay;
      oz.dL[1 + c] *= k.fdecay;
    }
  }
}

// Cell corrector (glm_physics.jl:128-172): exact momentum response to the trial velocity
// increment and the analytically integrated drag work removed from E, with the density
// floored at smallr and E floored at the new kinetic + magnetic energy + 1e-30. With `rE`
// the work is removed through E's Kahan remainder, which is cleared when the floor applies
// (drag_correct_conserved_compensated!, glm_physics.jl:374-400 with
// _compensated_floor_update!, :361-372).
__device__ __forceinline__ void drag_correct_cell(const F9& u0, F9& t, const DragCoef& k, float smallr,
                                                  float* rE = nullptr) {
  const float rn = fmaxf(t[0], smallr), ro = fmaxf(u0[0], smallr);
  float w[3], dv[3], vn[3], iw[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float vo = u0[1 + c] / ro, vt = t[1 + c] / rn;
    dv[c] = vt - vo;
    w[c] = vo - k.v0[c];
    vn[c] = k.v0[c] + k.decay * w[c] + k.phi1 * dv[c];
    iw[c] = (1.0f - k.decay) * w[c] + (1.0f - k.phi1) * dv[c];
  }
  const float w2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  const float wdv = w[0] * dv[0] + w[1] * dv[1] + w[2] * dv[2];
  const float dv2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
  const float qwork =
      rn * (k.A * w2 + k.C * wdv + k.D * dv2 + k.v0[0] * iw[0] + k.v0[1] * iw[1] + k.v0[2] * iw[2]);
  const float nm0 = rn * vn[0], nm1 = rn * vn[1], nm2 = rn * vn[2];
  const float ek = 0.5f * (nm0 * nm0 + nm1 * nm1 + nm2 * nm2) / rn;
  const float eb = 0.5f * (t[5] * t[5] + t[6] * t[6] + t[7] * t[7]);
  t[0] = rn;
  t[1] = nm0;
  t[2] = nm1;
  t[3] = nm2;
  const float emin = ek + eb + 1e-30f;
  if (rE == nullptr) {
    t[4] = fmaxf(t[4] - qwork, emin);
  } else {
    float e = comp_add(t[4], -qwork, *rE);
    if (e < emin) {
      *rE = 0.0f;
      e = emin;
    }
    t[4] = e;
  }
}

// Admissibility of a trial conserved state (integrator_cube.jl:108-124): finite, density
// at least max(smallr, llf_dmin) and internal energy at least pfl/(gamma-1).
__device__ __forceinline__ bool inadmissible_cell(const F9& r, const Phys& P) {
  const float ir = 1.0f / fmaxf(r[0], P.smallr);
  const float ek = 0.5f * (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) * ir;
  const float eb = 0.5f * (r[5] * r[5] + r[6] * r[6] + r[7] * r[7]);
  const float eint = r[4] - ek - eb;
  bool finite = isfinite(eint);
#pragma unroll
  for (int v = 0; v < 9; ++v) finite = finite && isfinite(r[v]);
  return !finite || r[0] < fmaxf(P.smallr, P.llf_dmin) || eint < P.pfl / (P.gamma - 1.0f);
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
