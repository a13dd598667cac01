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
template <int NL>
__device__ __forceinline__ void b_vdiff(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const float* ds = tb + m.to.dsigma;
  const float* sh = tb + m.to.sigmah;
  const float D2 = P.deltsec2;
  // Every field value used is read here, before the first store (the
  // compiler cannot prove the fields distinct, so a store would order each
  // later load after it). Within a full step only surflx's lowest level of
  // the tendencies holds more than physics_in's zeros (Model::zero_gdt).
  float zt[NL], zq[NL], zu[NL], zv[NL], zabsu[NL], zskap[NL], zskaph[NL];
  float dtdt[NL], dqdt[NL], dudt[NL], dvdt[NL], dq[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    const bool held = m.zero_gdt || l == NL - 1;
    dtdt[l] = held ? F.dtdt[at] : 0.f;
    dqdt[l] = held ? F.dqdt[at] : 0.f;
    dudt[l] = held ? F.dudt[at] : 0.f;
    dvdt[l] = held ? F.dvdt[at] : 0.f;
    dq[l] = F.dq[at];
    zt[l] = F.dt[at] + dtdt[l] * D2;
    zq[l] = dq[l] + dqdt[l] * D2;
    zu[l] = F.du[at] + dudt[l] * D2;
    zv[l] = F.dv[at] + dvdt[l] * D2;
    zabsu[l] = sqrtf(zu[l] * zu[l] + zv[l] * zv[l]);
    zskap[l] = tb[m.to.vdiff_skap + l];
    zskaph[l] = tb[m.to.vdiff_skaph + l];
  }
  const float zkonst1 = K.GA * D2 / K.GASCON;
  const float zkonst2 = zkonst1 * K.GA / K.GASCON;
  const float zkonst3 = zkonst2 * K.GA / K.GASCON;
  const float moisture = 1.f / K.RDBRV - 1.f;
  float kh[NL], km[NL];
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
        (zt[l] * (1.f + moisture * zq[l]) / zskap[l] - zt[lp] * (1.f + moisture * zq[lp]) / zskap[lp]) * zrdsig;
    const float zri = zskaph[l] * K.GASCON * zdthds / (sigmah * zdvds * zdvds);
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
  float zun[NL], zvn[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    zun[l] = zu[l];
    zvn[l] = zv[l];
  }
  diffuse<NL>(ds, zun, km);
  diffuse<NL>(ds, zvn, km);
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    F.dudt[at] = dudt[l] + __fdiv_rn(zun[l] - zu[l], D2);
    F.dvdt[at] = dvdt[l] + __fdiv_rn(zvn[l] - zv[l], D2);
  }
  if (K.NDHEAT != 0.f) {
    float zke[NL], zken[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) zke[l] = zken[l] = 0.5f * zabsu[l] * zabsu[l];
    diffuse<NL>(ds, zken, km);
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      const float zdtdt = -((zun[l] * zun[l] - zu[l] * zu[l] + zvn[l] * zvn[l] - zv[l] * zv[l]) / D2 -
                            (zken[l] - zke[l]) / D2) * 0.5f / K.ACPD / (1.f + K.ADV * dq[l]);
      dtdt[l] = dtdt[l] + zdtdt;
    }
  }
  float zqn[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) zqn[l] = zq[l];
  diffuse<NL>(ds, zqn, kh);
#pragma unroll
  for (int l = 0; l < NL; ++l) F.dqdt[l * SN + c] = dqdt[l] + __fdiv_rn(zqn[l] - zq[l], D2);
#pragma unroll
  for (int l = 0; l < NL - 1; ++l) kh[l] = kh[l] * zskaph[l];
  float ztn[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) ztn[l] = zt[l];
  diffuse_potential<NL>(ds, ztn, kh, zskap);
#pragma unroll
  for (int l = 0; l < NL; ++l) F.dtdt[l * SN + c] = dtdt[l] + __fdiv_rn(ztn[l] - zt[l], D2);
}
template <int NL>
__global__ void __launch_bounds__(kBlock, 3) k_vdiff(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_vdiff<NL>(m, pcr, tabr);
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
COLUMN_LAUNCHER(Vdiff, k_vdiff)
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
