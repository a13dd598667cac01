// The fixer's apply step, the surface fluxes and vertical diffusion, and the
// solar angle and ozone columns. vdiff's tendencies are small differences of
// two implicitly diffused profiles, so its tridiagonal solves
// (physics_common.cuh) and the tendency quotients divide to IEEE precision
// (__fdiv_rn); with 2-ulp quotients there, more points of its humidity
// tendency left the reference's V3 tolerance than a sequential-f32 build's.
// Arithmetic follows physics/fixer/wgsl/apply.wgsl, physics/surface-flux/
// wgsl/{surflx,vdiff}.wgsl, physics/diffusion/wgsl/implicit.wgsl and
// physics/radiation/wgsl/{solang,mko3}.wgsl; a full step runs the four as
// one fused column kernel, stage replay as four launches.
#include "physics_common.cuh"

namespace exogcm {

namespace {

// physics/fixer/wgsl/apply.wgsl: the global step, gqdt and the new dq. The
// fixer is the first to raise gqdt after physics_in zeroed it, so within a
// full step (Model::zero_gdt = 0) it adds its increment to 0 unread.
template <int NL>
__device__ __forceinline__ void b_fixer_apply(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const double zzneg = m.sums[slot * 4], zzpos = m.sums[slot * 4 + 1];
  const float scale = zzneg > 0.0 ? (float)((zzpos - zzneg) / zzpos) : 1.f;
  const float dp = F.dp[c];
  // every level's inputs are read before the first store (the compiler
  // cannot prove the fields distinct)
  float fq[NL], gq[NL], dq[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    fq[l] = F.fixq[at];
    gq[l] = m.zero_gdt ? F.gqdt[at] : 0.f;
    dq[l] = F.dq[at];
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    float q = fq[l];
    if (zzneg > 0.0) q = fmaxf(q * scale, 0.f);
    F.gqdt[at] = gq[l] + dp * (q - dq[l]) / P.delt2 / K.PSURF;
    F.dq[at] = q;
  }
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_fixer_apply(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_fixer_apply<NL>(m, pcr, tabr);
}


// ---------------------------------------------------------------- surface flux
// physics/surface-flux/wgsl/surflx.wgsl: transfer coefficients, implicit
// stress, sensible heat and evaporation.
template <int NL>
__device__ __forceinline__ void b_surflx(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const int low = NL - 1;
  const size_t lo = low * SN + c, sf = NL * SN + c;
  const float u = F.du[lo], v = F.dv[lo], t = F.dt[lo], q = F.dq[lo], ts = F.dt[sf], qs = F.dq[sf];
  const float dp = F.dp[c], dls = F.dls[c];
  // the tendencies and surface values used after the first store are read
  // here (the compiler cannot prove the fields distinct); within a full step
  // the tendencies hold physics_in's zeros, taken unread (Model::zero_gdt)
  const bool earlier = m.zero_gdt != 0;
  const float dudt0 = earlier ? F.dudt[lo] : 0.f, dvdt0 = earlier ? F.dvdt[lo] : 0.f;
  const float dtdt0 = earlier ? F.dtdt[lo] : 0.f, dqdt0 = earlier ? F.dqdt[lo] : 0.f;
  const float drhs = F.drhs[c], dwatc = F.dwatc[c], dz0 = F.dz0[c];
  const float dsigma = tb[m.to.dsigma + low];
  const float zfac = tb[m.to.flux_sigfac], zlnsig = tb[m.to.flux_lnsig];
  const float moisture = 1.f / K.RDBRV - 1.f;
  const float VK = 0.4f;
  const float D2 = P.deltsec2;
  float dtsa = t * zfac * (1.f + moisture * q);
  const float zabsu2 = fmaxf(K.ZUMIN, u * u + v * v);
  const float znl = -K.GASCON * 0.5f * (t + dtsa) * zlnsig / K.GA;
  const float zbz0 = znl / dz0;
  const float zri = K.GA * znl / (zabsu2 * dtsa) * (dtsa - ts * (1.f + moisture * qs));
  const float zkblnz = VK / logf(zbz0 + 1.f);
  const float zkblnz2 = zkblnz * zkblnz;
  float zrifm, zrifh;
  if (zri <= 0.f) {
    const float zdenom = 1.f + 3.f * K.VDIFF_C * K.VDIFF_B * sqrtf(-1.f * zri * (zbz0 + 1.f)) * zkblnz2;
    zrifm = 1.f - 2.f * K.VDIFF_B * zri / zdenom;
    if (dls < 1.f) {
      const float zdth = -(dtsa - ts * (1.f + moisture * qs));
      zrifh = powf(1.f + powf(0.0016f * powf(zdth, 1.f / 3.f) / sqrtf(zabsu2) / zkblnz2, 1.25f), 0.8f);
    } else {
      zrifh = 1.f - 3.f * K.VDIFF_B * zri / zdenom;
    }
  } else {
    const float zdenom = sqrtf(1.f + K.VDIFF_D * zri);
    zrifh = 1.f / (1.f + 3.f * K.VDIFF_B * zri * zdenom);
    zrifm = 1.f / (1.f + 2.f * K.VDIFF_B * zri / zdenom);
  }
  const float ztrans = sqrtf(zabsu2) * zkblnz2;
  const float transh = ztrans * zrifh, transm = ztrans * zrifm;
  F.dtransh[c] = transh;
  F.dtransm[c] = transm;
  const float zkonst1 = K.GA * D2 / (K.GASCON * dsigma);
  const float zkonst2 = dsigma / D2 / K.GA;
  const float zkdiffm = zkonst1 * transm / ts;
  const float zun = u / (1.f + zkdiffm), zvn = v / (1.f + zkdiffm);
  F.dudt[lo] = dudt0 + (zun - u) / D2;
  F.dvdt[lo] = dvdt0 + (zvn - v) / D2;
  float dtdt = dtdt0;
  if (K.NDHEAT != 0.f) dtdt = dtdt + -(zun * zun - u * u + zvn * zvn - v * v) / D2 * 0.5f / K.ACPD / (1.f + K.ADV * q);
  const float taux = dp * zkonst2 * zkdiffm * zun, tauy = dp * zkonst2 * zkdiffm * zvn;
  F.dtaux[c] = taux;
  F.dtauy[c] = tauy;
  const float ustar = sqrtf(sqrtf(taux * taux + tauy * tauy) * K.GASCON * ts / dp);
  F.dust3[c] = ustar * ustar * ustar;
  const float zkdiffh = zkonst1 * transh / ts;
  const float ztn = (t + zkdiffh * ts) / (1.f + zkdiffh * zfac);
  dtdt = dtdt + (ztn - t) / D2;
  F.dtdt[lo] = dtdt;
  const float moist = fmaxf(1.f, 1.f + K.ADV * q);
  F.dshfl[c] = zkonst2 * zkdiffh * dp * K.ACPD * moist * (ztn * zfac - ts);
  F.dshdt[c] = -1.f * zkonst2 * zkdiffh * dp * K.ACPD * moist;
  dtsa = ztn * zfac;
  F.dtsa[c] = dtsa;
  const float zkdiffq = drhs * zkonst1 * transh / ts;
  float zqn = fmaxf(q, (q + zkdiffq * qs) / (1.f + zkdiffq));
  if (dls > 0.f) zqn = fminf(zqn, dwatc / P.deltsec * 1000.f / dp / zkonst2 + q);
  F.dqdt[lo] = dqdt0 + (zqn - q) / D2;
  const float devap = -dp * zkonst2 / 1000.f * (zqn - q);
  F.devap[c] = devap;
  const float latent = (ts > K.TMELT || dls < 0.5f) ? K.ALV : K.ALS;
  const float dlhfl = devap * latent * 1000.f;
  F.dlhfl[c] = dlhfl;
  const float curvature = (ts - K.RA4) * (ts - K.RA4);
  const float dlhdt = -1.f * latent * zkdiffq * zkonst2 * dp * K.RA2 * (K.TMELT - K.RA4) * qs / curvature;
  F.dlhdt[c] = dlhfl == 0.f ? 0.f : dlhdt;
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_surflx(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_surflx<NL>(m, pcr, tabr);
}


// physics/diffusion/wgsl/implicit.wgsl: ECHAM tridiagonal eliminations.
// physics/surface-flux/wgsl/vdiff.wgsl: Richardson-number vertical diffusion.
// HOLD: which levels of the tendencies dtdt, dqdt, dudt, dvdt hold values on
// entry: 1 every level (stage replay, Model::zero_gdt), 0 only the lowest
// (within a full step, where physics_in's zeros are taken as values and
// surflx raised the lowest level), -1 decided at run time from zero_gdt.
// With HOLD = 0 the other levels' tendencies are the constant 0 and need no
// registers.
// |(u, v)| with both squares rounded before the sum (no contraction), the
// same wherever the speed is formed.
__device__ __forceinline__ float wind_speed(float u, float v) {
  return sqrtf(__fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v)));
}

template <int NL, int HOLD = -1>
__device__ __forceinline__ void b_vdiff(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const float* ds = tb + m.to.dsigma;
  const float* sh = tb + m.to.sigmah;
  const float* skap = tb + m.to.vdiff_skap;
  const float* skaph = tb + m.to.vdiff_skaph;
  const float D2 = P.deltsec2;
  const bool all_held = HOLD < 0 ? m.zero_gdt != 0 : HOLD == 1;
  // An incoming tendency: every level in stage replay; within a full step
  // only the lowest holds more than physics_in's zeros (Model::zero_gdt).
  auto tend = [&](const float* f, int l) { return all_held || l == NL - 1 ? f[l * SN + c] : 0.f; };
  // The routine runs in three phases so that few level columns are live at
  // once: the exchange coefficients, then humidity and temperature (whose
  // profiles are then dropped), then the winds and the dissipative heating,
  // whose inputs are read again (no field read here is written here). Each
  // value is computed by the same expression as in one pass.
  float zt[NL], zq[NL], kh[NL], km[NL];
  {
    float zabsu[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const size_t at = l * SN + c;
      zt[l] = F.dt[at] + tend(F.dtdt, l) * D2;
      zq[l] = F.dq[at] + tend(F.dqdt, l) * D2;
      const float zu = F.du[at] + tend(F.dudt, l) * D2;
      const float zv = F.dv[at] + tend(F.dvdt, l) * D2;
      zabsu[l] = wind_speed(zu, zv);
    }
    const float zkonst1 = K.GA * D2 / K.GASCON;
    const float zkonst2 = zkonst1 * K.GA / K.GASCON;
    const float zkonst3 = zkonst2 * K.GA / K.GASCON;
    const float moisture = 1.f / K.RDBRV - 1.f;
    kh[NL - 1] = 0.f;
    km[NL - 1] = 0.f;
#pragma unroll
    for (int l = 0; l < NL - 1; ++l) {
      const int lp = l + 1;
      const float sigmah = sh[l], dsigma = ds[l], dsigmap = ds[lp];
      const float zmixh2 = tb[m.to.vdiff_mixh2 + l], zmixm2 = tb[m.to.vdiff_mixm2 + l];
      const float zrdsig = tb[m.to.vdiff_rdsig + l];
      const float zfac = zkonst3 * tb[m.to.vdiff_sigmah3 + l];
      const float zzkfac = tb[m.to.vdiff_kfac + l];
      const float zrthl = (dsigmap + dsigma) / (zt[l] * dsigmap + zt[lp] * dsigma);
      const float zdvds = fmaxf(K.ZUMIN, fabsf(zabsu[l] - zabsu[lp])) * zrdsig;
      const float zdthds =
          (zt[l] * (1.f + moisture * zq[l]) / skap[l] - zt[lp] * (1.f + moisture * zq[lp]) / skap[lp]) * zrdsig;
      const float zri = skaph[l] * K.GASCON * zdthds / (sigmah * zdvds * zdvds);
      float zrifh, zrifm;
      if (zri <= 0.f) {
        const float dh = 1.f + 3.f * K.VDIFF_C * K.VDIFF_B * sqrtf(-1.f * zri) * zzkfac * zmixh2;
        const float dm = 1.f + 3.f * K.VDIFF_C * K.VDIFF_B * sqrtf(-1.f * zri) * zzkfac * zmixm2;
        zrifh = 1.f - 3.f * K.VDIFF_B * zri / dh;
        zrifm = 1.f - 2.f * K.VDIFF_B * zri / dm;
      } else {
        const float zdenom = sqrtf(1.f + K.VDIFF_D * zri);
        zrifh = 1.f / (1.f + 3.f * K.VDIFF_B * zri * zdenom);
        zrifm = 1.f / (1.f + 2.f * K.VDIFF_B * zri / zdenom);
      }
      kh[l] = zfac * zmixh2 * zrifh * zdvds * zrthl * zrthl * zrthl;
      km[l] = zfac * zmixm2 * zrifm * zdvds * zrthl * zrthl * zrthl;
    }
  }
  // humidity, stored at once
  {
    float zqn[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) zqn[l] = zq[l];
    diffuse<NL>(ds, zqn, kh);
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const size_t at = l * SN + c;
      F.dqdt[at] = tend(F.dqdt, l) + __fdiv_rn(zqn[l] - zq[l], D2);
    }
  }
  // temperature: its diffusion increment, stored with the heating below
  float zdt[NL];
  {
    float zskap[NL], ztn[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      zskap[l] = skap[l];
      ztn[l] = zt[l];
    }
#pragma unroll
    for (int l = 0; l < NL - 1; ++l) kh[l] = kh[l] * skaph[l];
    diffuse_potential<NL>(ds, ztn, kh, zskap);
#pragma unroll
    for (int l = 0; l < NL; ++l) zdt[l] = __fdiv_rn(ztn[l] - zt[l], D2);
  }
  // winds and the dissipative heating
  float zu[NL], zv[NL], zun[NL], zvn[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    zu[l] = F.du[at] + tend(F.dudt, l) * D2;
    zv[l] = F.dv[at] + tend(F.dvdt, l) * D2;
    zun[l] = zu[l];
    zvn[l] = zv[l];
  }
  diffuse<NL>(ds, zun, km);
  diffuse<NL>(ds, zvn, km);
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    F.dudt[at] = tend(F.dudt, l) + __fdiv_rn(zun[l] - zu[l], D2);
    F.dvdt[at] = tend(F.dvdt, l) + __fdiv_rn(zvn[l] - zv[l], D2);
  }
  float heat[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) heat[l] = tend(F.dtdt, l);
  if (K.NDHEAT != 0.f) {
    float zke[NL], zken[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const float zabsu = wind_speed(zu[l], zv[l]);
      zke[l] = zken[l] = 0.5f * zabsu * zabsu;
    }
    diffuse<NL>(ds, zken, km);
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const float dq = F.dq[l * SN + c];
      // zun^2 - zu^2 + zvn^2 - zv^2 left to right; the squares of the winds
      // before diffusion are rounded on their own
      const float uu = __fmul_rn(zu[l], zu[l]), vv = __fmul_rn(zv[l], zv[l]);
      const float dke = __fsub_rn(__fmaf_rn(zvn[l], zvn[l], __fmaf_rn(zun[l], zun[l], -uu)), vv);
      const float zdtdt = -(dke / D2 - (zken[l] - zke[l]) / D2) * 0.5f / K.ACPD / (1.f + K.ADV * dq);
      heat[l] = heat[l] + zdtdt;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) F.dtdt[l * SN + c] = heat[l] + zdt[l];
}
template <int NL, int HOLD>
__global__ void __launch_bounds__(kBlock, HOLD == 0 ? 4 : 3)
    k_vdiff(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_vdiff<NL, HOLD>(m, pcr, tabr);
}



// solang (physics/radiation/wgsl/solang.wgsl) and mko3 (mko3.wgsl) for one column.
template <int NL>
__device__ __forceinline__ void b_solang_mko3(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const int lat = h / d.NLON, lon = h % d.NLON;
  float hangle = P.rad[2] + (float)lon * K.ZRLON - kPI;
  if (hangle < -kPI) hangle = hangle + kTWOPI;
  if (hangle > kPI) hangle = hangle - kTWOPI;
  if (K.NFIXED == 1.f) hangle = hangle + kPI;
  const float muz = P.rad[0] * m.sh.sid[lat] + m.sh.cola[lat] * P.rad[1] * cosf(hangle);
  F.gmu0[c] = muz > K.ZDAWN ? muz : 0.f;
  if (K.OZONE == 0.f) return;
  const float ZFO3 = 100.f / 2.14f;
  const float sid = m.sh.sid[lat];
  const float za = K.A0O3 + K.A1O3 * fabsf(sid) + K.ACO3 * sid * P.rad[4];
  const float dp = F.dp[c];
  const float* ds = tb + m.to.dsigma;
  const float* lnsig = tb + m.to.rad_lnsig;
  float o3t = za, zh = 0.f;
  float t[NL];  // read before the stores below (possible aliasing would order them)
#pragma unroll
  for (int l = 1; l < NL; ++l) t[l] = F.dt[l * SN + c];
#pragma unroll
  for (int l = NL - 1; l >= 1; --l) {
    zh = zh - t[l] * K.GASCON / K.GA * lnsig[l];
    const float o3 = -(za + za * K.ZCONST) / (1.f + expf((zh - K.BO3) / K.CO3)) + o3t;
    F.dqo3[l * SN + c] = o3 * K.GA / (ZFO3 * ds[l] * dp);
    o3t = o3t - o3;
  }
  F.dqo3[c] = o3t * K.GA / (ZFO3 * ds[0] * dp);
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_solang_mko3(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_solang_mko3<NL>(m, pcr, tabr);
}



// The full step's fused kernel: fixer apply, surface fluxes, vertical
// diffusion, solar angle and ozone for one column per thread.
template <int NL>
__global__ void __launch_bounds__(kBlock, 3) k_fused_fixer_flux_solang(Model m, const PlanetConst* __restrict__ pcr,
                                                                       const float* __restrict__ tabr) {
  b_fixer_apply<NL>(m, pcr, tabr);
  b_surflx<NL>(m, pcr, tabr);
  b_vdiff<NL>(m, pcr, tabr);
  b_solang_mko3<NL>(m, pcr, tabr);
}

COLUMN_LAUNCHER(FixerApply, k_fixer_apply)
COLUMN_LAUNCHER(Surflx, k_surflx)
template <int NL>
struct Vdiff {
  static void run(const Model& m, cudaStream_t st) {
    const unsigned blocks = nblocks((size_t)m.d.S * m.d.NHOR, kBlock);
    if (m.zero_gdt)
      pdl_launch(k_vdiff<NL, 1>, blocks, kBlock, 0, st, m, m.pc, m.tabs);
    else
      pdl_launch(k_vdiff<NL, 0>, blocks, kBlock, 0, st, m, m.pc, m.tabs);
  }
};
COLUMN_LAUNCHER(SolangMko3, k_solang_mko3)
COLUMN_LAUNCHER(FusedFixerFluxSolang, k_fused_fixer_flux_solang)

}  // namespace

void phy_fixer_apply(const Model& m, cudaStream_t st) { by_levels<FixerApply>(m.d.L, m, st); }

void phy_surface_flux(const Model& m, cudaStream_t st) {
  by_levels<Surflx>(m.d.L, m, st);
  by_levels<Vdiff>(m.d.L, m, st);
}

void phy_solang_mko3(const Model& m, cudaStream_t st) { by_levels<SolangMko3>(m.d.L, m, st); }

void phy_fused_fixer_flux_solang(const Model& m, cudaStream_t st) {
  by_levels<FusedFixerFluxSolang>(m.d.L, m, st);
}

bool phy_flux_launch_one(const Model& m, const std::string& kernel, cudaStream_t st) {
  if (kernel == "vdiff") by_levels<Vdiff>(m.d.L, m, st);
  else if (kernel == "surflx") by_levels<Surflx>(m.d.L, m, st);
  else if (kernel == "fixer_apply") by_levels<FixerApply>(m.d.L, m, st);
  else if (kernel == "solang_mko3") by_levels<SolangMko3>(m.d.L, m, st);
  else if (kernel == "fused_fixer_flux_solang") by_levels<FusedFixerFluxSolang>(m.d.L, m, st);
  else return false;
  return true;
}

}  // namespace exogcm
