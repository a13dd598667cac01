// hurricanestep: the storm-climatology diagnostics of one column
// (physics/storm/wgsl/storm.wgsl:1-208, after ExoPlaSim's hurricanemod.f90),
// run after carbonstep and before the frame out when a planet enables them
// (NSTORMDIAG, hurricane_namelist; physics/storm/index.ts:26-43).
//
// One thread per column in FP32. This file keeps CUDA's accurate exp, log,
// pow and IEEE division: the saturated-parcel and pressure solvers iterate
// to fixed tolerances, so a coarser step changes their iteration counts.
//
// The reference's WGSL pow(x, y) is undefined for x < 0; the genesis index
// raises 2 RH to the third power, and RH at the level nearest sigma 0.6 is
// negative when the model's humidity there is. powf follows the native
// Fortran's x**3.0 there (a negative cube), where a WGSL implementation's
// exp2(y log2 x) gives NaN.
#include "launch.h"
#include "physics_common.cuh"

namespace exogcm {
namespace {

// hurricanemod.f90's fixed thermodynamic constants (storm.wgsl:6-11).
constexpr float kCpd = 1005.7f;
constexpr float kCl = 2500.0f;
constexpr float kRvp = 461.5f;
constexpr float kAlv0 = 2.501e6f;
constexpr float kCpvmcl = -630.0f;

struct Cape {
  float energy, temperature, pressure;
};

// Saturation vapour pressure (hPa) at tc degrees Celsius.
__device__ __forceinline__ float es(float tc) { return 6.112f * expf(17.67f * tc / (243.5f + tc)); }

// Vapour pressure from mixing ratio r at pressure p.
__device__ __forceinline__ float vapor(float r, float p, float rd) { return r * p / (rd / kRvp + r); }

// Mixing ratio from vapour pressure e at pressure p.
__device__ __forceinline__ float mixing(float e, float p, float rd) { return (rd / kRvp) * e / (p - e); }

// Density temperature of temperature t, total water rt and vapour r.
__device__ __forceinline__ float density(float t, float rt, float r, float rd) {
  return t * (1.0f + r / (rd / kRvp)) / (1.0f + rt);
}

// Moist entropy of temperature t, mixing ratio r and pressure p.
__device__ __forceinline__ float entropy(float t, float r, float p, float rd) {
  const float e = vapor(r, p, rd);
  const float rh = fminf(e / es(t - 273.15f), 1.0f);
  const float lv = kAlv0 + kCpvmcl * (t - 273.15f);
  const float dry = (kCpd + r * kCl) * logf(t) - rd * logf(p - e);
  if (r == 0.0f) return dry;
  return dry + lv * r / t - r * kRvp * logf(rh);
}

// Reversible-ascent CAPE of the parcel (tp, rp, pp) through the sounding
// (storm.wgsl:56-126): levels top (0) to bottom (NL - 1).
template <int NL>
__device__ Cape cape(const float (&st)[NL], const float (&sr)[NL], const float (&sp)[NL], float tp, float rp,
                     float pp, float rd) {
  if (rp < 1e-6f || tp < 200.0f || pp <= 0.0f) return {0.0f, -1.0f, -1.0f};
  const float rh = fminf(vapor(rp, pp, rd) / es(tp - 273.15f), 1.0f);
  const float parcel_entropy = entropy(tp, rp, pp, rd);
  const float plcl = pp * powf(rh, tp / (1669.0f - 122.0f * rh - tp));
  float buoyancy[NL];
  for (int l = NL - 1; l >= 0; --l) {
    float tg, rg = rp;
    if (sp[l] >= plcl) {
      tg = tp * powf(sp[l] / pp, rd / kCpd);
    } else {
      // Saturated ascent: Newton steps on the parcel's entropy, 0.3 of a
      // step for the first two, until the temperature moves by 0.001 K.
      float next = st[l];
      tg = 0.0f;
      int count = 0;
      while (!(fabsf(next - tg) <= 0.001f)) {
        tg = next;
        const float tc = tg - 273.15f;
        const float enew = es(tc);
        rg = mixing(enew, sp[l], rd);
        ++count;
        const float lv = kAlv0 + kCpvmcl * tc;
        const float sl = (kCpd + rp * kCl + lv * lv * rg / (kRvp * tg * tg)) / tg;
        const float em = vapor(rg, sp[l], rd);
        if (sp[l] - em <= 0.0f || tg <= 0.0f) return {0.0f, st[l], -1.0f};
        const float sg = (kCpd + rp * kCl) * logf(tg) - rd * logf(sp[l] - em) + lv * rg / tg;
        next = tg + (count < 3 ? 0.3f : 1.0f) * (parcel_entropy - sg) / sl;
        if (count > 500 || enew > sp[l] - 1.0f || !(next > 0.0f)) return {0.0f, st[NL - 1], sp[NL - 1]};
      }
    }
    buoyancy[l] = density(tg, rp, rg, rd) - density(st[l], sr[l], sr[l], rd);
  }
  int inb = NL - 1;
#pragma unroll
  for (int l = 0; l < NL; ++l)
    if (buoyancy[l] > 0.0f) inb = min(inb, l);
  if (inb == NL - 1) return {0.0f, st[NL - 1], 0.0f};
  float area = 0.0f;
#pragma unroll
  for (int l = NL - 2; l >= 0; --l)
    if (l >= inb) area += rd * (buoyancy[l] + buoyancy[l + 1]) * (sp[l + 1] - sp[l]) / (sp[l] + sp[l + 1]);
  area += rd * (pp - sp[NL - 1]) / (pp + sp[NL - 1]) * buoyancy[NL - 1];
  float tob = st[inb], lnb = sp[inb];
  if (inb > 0) {
    const float b0 = buoyancy[inb - 1], b1 = buoyancy[inb];
    lnb = (sp[inb - 1] * b1 - sp[inb] * b0) / (b1 - b0);
    area += rd * b1 * (sp[inb] - lnb) / (sp[inb] + lnb);
    tob = (st[inb] * (lnb - sp[inb - 1]) + st[inb - 1] * (sp[inb] - lnb)) / (sp[inb] - sp[inb - 1]);
  }
  return {fmaxf(area, 0.0f), tob, lnb};
}

// Real part of the principal cube root in hurricanemod's ventilation-
// reduced intensity: zero at VI = 0 and for |VI| >= VITHRESH.
__device__ __forceinline__ float reduced(float vi, float vithresh) {
  if (vi == 0.0f || fabsf(vi) >= vithresh) return 0.0f;
  return 2.0f / sqrtf(3.0f) * cosf(acosf(-vi / vithresh) / 3.0f);
}

template <int NL>
__global__ void __launch_bounds__(kBlock) k_storm(Model m, const PlanetConst* __restrict__ pcr,
                                                  const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  if (K.NSTORMDIAG <= 0.0f) return;
  const float* sg = tb + m.to.sigma;
  const float rd = K.GASCON;
  float st[NL], sr[NL], sp[NL];
  const float msl = F.dp[c] * 0.01f;
  const float sst = F.dt[NL * SN + c];
  int i600 = 0, i850 = 0, i200 = 0;
  bool cold = false;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    st[l] = F.dt[l * SN + c];
    sr[l] = F.dq[l * SN + c];
    sp[l] = msl * sg[l];
    cold = cold || st[l] <= 100.0f;
    if (fabsf(sg[l] - 0.6f) < fabsf(sg[i600] - 0.6f)) i600 = l;
    if (fabsf(sg[l] - 0.85f) < fabsf(sg[i850] - 0.85f)) i850 = l;
    if (fabsf(sg[l] - 0.2f) < fabsf(sg[i200] - 0.2f)) i200 = l;
  }
  constexpr int bottom = NL - 1;
  const float u850 = F.du[i850 * SN + c], v850 = F.dv[i850 * SN + c];
  const float u200 = F.du[i200 * SN + c], v200 = F.dv[i200 * SN + c];
  const float lowwind = sqrtf(u850 * u850 + v850 * v850), highwind = sqrtf(u200 * u200 + v200 * v200);
  const float shear = fabsf(highwind - lowwind);
  const float vort = F.gz[i850 * SN + c] * K.WW;
  float deficit = 1.0f;
  if (sr[i600] > 0.0f && sr[bottom] > 0.0f) {
    const float smr = mixing(es(st[i600] - 273.15f), sp[i600], rd);
    const float sms = entropy(st[i600], smr, sp[i600], rd);
    const float sme = entropy(st[i600], fminf(sr[i600], smr), sp[i600], rd);
    const float smb = entropy(sst, F.dq[NL * SN + c], msl, rd);
    const float smo = entropy(sst, mixing(es(sst - 273.15f), msl, rd), msl, rd);
    if (smo != smb) deficit = (sms - sme) / (smo - smb);
  }
  Cape environmental{-1.0f, -1.0f, -1.0f};
  float vmax = -1.0f;
  if (sst > 278.15f && !cold && msl > 0.0f) {
    environmental = cape<NL>(st, sr, sp, st[bottom], sr[bottom], sp[bottom], rd);
    // Minimum central pressure: 970 hPa first, 1000 hPa parcel cap, until
    // it moves by 0.5 hPa; bail out after 201 passes or below 400 hPa.
    float pm = 970.0f, old = pm, next = 0.0f, capem = 0.0f, capems = 0.0f, ratio = 1.0f;
    bool failed = false;
    int count = 0;
    while (!(fabsf(next - old) <= 0.5f)) {
      const float pp = fminf(pm, 1000.0f);
      const float rp = (rd / kRvp) * sr[bottom] * msl / (pp * (rd / kRvp + sr[bottom]) - sr[bottom] * msl);
      capem = cape<NL>(st, sr, sp, st[bottom], rp, pp, rd).energy;
      const float rs = mixing(es(sst - 273.15f), pp, rd);
      const Cape saturated = cape<NL>(st, sr, sp, sst, rs, pp, rd);
      capems = saturated.energy;
      ratio = sst / saturated.temperature;
      const float tvav = 0.5f * (density(st[bottom], sr[bottom], sr[bottom], rd) + density(sst, rs, rs, rd));
      const float cat = fmaxf((capem - environmental.energy) + 0.5f * K.CKCD * ratio * (capems - capem), 0.0f);
      next = msl * expf(-cat / (rd * tvav));
      old = pm;
      pm = next;
      ++count;
      if (count > 200 || pm < 400.0f || !(pm > 0.0f)) {
        failed = true;
        break;
      }
    }
    if (!failed) vmax = sqrtf(fmaxf(0.0f, K.CKCD * ratio * fmaxf(0.0f, capems - capem)));
  }
  const float vi = vmax > 0.0f ? shear * deficit / vmax : 1.0f;
  const float rh = vapor(sr[i600], sp[i600], rd) / es(st[i600] - 273.15f);
  const float v70 = vmax / 70.0f, damp = 1.0f + 0.1f * shear;
  const float gpi = powf(fabsf(vort * 1e5f), 1.5f) * powf(rh * 2.0f, 3.0f) * v70 * v70 * v70 / (damp * damp);
  F.capen[c] = environmental.energy;
  F.lnb[c] = environmental.pressure;
  F.mpoti[c] = vmax;
  F.chim[c] = deficit;
  F.laav[c] = vort;
  F.venti[c] = vi;
  F.vrmpi[c] = reduced(vi, K.VITHRESH);
  F.gpi[c] = gpi;
  F.shear[c] = shear;
}

COLUMN_LAUNCHER(Storm, k_storm)

}  // namespace

void phy_storm(const Model& m, cudaStream_t st) {
  if (!m.storm) return;
  by_levels<Storm>(m.d.L, m, st);
}

}  // namespace exogcm
