// Grid-point dynamics, semi-implicit spectral update, horizontal diffusion,
// dissipative heating and the dimensional frame around the column physics,
// for every slot of a batch in one launch each (FP32).
//
// Arithmetic follows src/model/climate/gcm/dynamics/wgsl/*.wgsl (ExoPlaSim
// plasim.f90's gridpointa / spectrala / spectrald / gridpointd, in Fortran's
// statement order), with the batch's [level][slot][point] layout: column
// index c = slot * NHOR + h, spectral index c = slot * NRSP + s.
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.h"

namespace exogcm {

namespace {

constexpr int kBlock = 128;

__device__ __forceinline__ const float* slot_tabs(const Model& m, int slot) {
  return m.tabs + (size_t)slot * m.to.stride;
}

// gridpointa from gp = exp(gp) to the flux products (dynamics/wgsl/calcgp.wgsl).
// Four resident blocks per SM: a few spilled registers cost less than the
// latency the fourth block hides.
template <int NL>
__global__ void __launch_bounds__(kBlock, 4) k_calcgp(Model m) {
  const Dims& d = m.d;
  // NHOR is a multiple of kBlock at every truncation, so a block lies in one
  // slot and that slot's vertical tables are staged in shared memory once.
  const int slot = blockIdx.x * kBlock / d.NHOR;
  if (!m.params[slot].active) return;
  __shared__ float stage[6 * NL + 2 * NL * NL];
  float* ds = stage;
  float* t0T = ds + NL;
  float* sh = t0T + NL;
  float* rd = sh + NL;
  float* t01 = rd + NL;
  float* tkpT = t01 + NL;
  float* C = tkpT + NL;
  float* G = C + NL * NL;
  {
    const float* tb = slot_tabs(m, slot);
    for (int i = threadIdx.x; i < NL * NL; i += kBlock) {
      C[i] = tb[m.to.c + i];
      G[i] = tb[m.to.g + i];
    }
    for (int i = threadIdx.x; i < NL; i += kBlock) {
      ds[i] = tb[m.to.dsigma + i];
      t0T[i] = tb[m.to.t0 + i];
      sh[i] = tb[m.to.sigmah + i];
      rd[i] = tb[m.to.rdsig + i];
      t01[i] = tb[m.to.t01s2 + i];
      tkpT[i] = tb[m.to.tkp + i];
    }
  }
  __syncthreads();
  const int c = blockIdx.x * kBlock + threadIdx.x;
  // The planet's constants are read once, before the first store (the
  // compiler cannot prove the fields distinct from them and would reload
  // each one after every store).
  const PlanetConst& Kg = m.pc[slot];
  struct {
    float AKAP, PSURF, WW, CV, RDBRV, ADV;
  } const K = {Kg.AKAP, Kg.PSURF, Kg.WW, Kg.CV, Kg.RDBRV, Kg.ADV};
  const size_t SN = (size_t)d.S * d.NHOR;
  const FieldPtrs& F = m.f;
  const float rcsq = m.sh.rcsq[c % d.NHOR];
  // gp = exp(gp) is stored with the first tendencies below, after every
  // load: a store here would hold back the loads that follow it.
  const float ps = expf(F.gp[c]);
  const float gpm = F.gpmt[c], gpj = F.gpj[c];
  float gu[NL], gv[NL], gt[NL], gd[NL], gz[NL], gq[NL], zvgpg[NL], ztv1[NL], ztv2[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    gu[l] = F.gu[at];
    gv[l] = F.gv[at];
    gt[l] = F.gt[at];
    gd[l] = F.gd[at];
    gz[l] = F.gz[at];
    gq[l] = F.gq[at];
    zvgpg[l] = rcsq * (gu[l] * gpm + gv[l] * gpj);
    const float zq = fmaxf(gq[l] / ps, 0.f);
    const float t0 = t0T[l];
    const float tvirt = (gt[l] + t0) * (1.f + (1.f / K.RDBRV - 1.f) * zq);
    ztv1[l] = tvirt - t0;
    ztv2[l] = tvirt / (1.f + K.ADV * zq) - t0;
  }
  float zsdotp[NL];
  float zsumd = ds[0] * gd[0];
  float gvp = ds[0] * zvgpg[0];
  zsdotp[0] = zsumd + gvp;
#pragma unroll
  for (int l = 1; l < NL - 1; ++l) {
    zsumd = zsumd + ds[l] * gd[l];
    gvp = gvp + ds[l] * zvgpg[l];
    zsdotp[l] = zsumd + gvp;
  }
  zsumd = zsumd + ds[NL - 1] * gd[NL - 1];
  gvp = gvp + ds[NL - 1] * zvgpg[NL - 1];
  float gtd[NL], gqm[NL], gud[NL], gvd[NL];
#pragma unroll
  for (int l = 0; l < NL - 1; ++l) {
    zsdotp[l] = sh[l] * (zsumd + gvp) - zsdotp[l];
    gtd[l] = zsdotp[l] * (gt[l + 1] - gt[l]);
    gqm[l] = zsdotp[l] * (gq[l + 1] + gq[l]);
    gud[l] = zsdotp[l] * (gu[l + 1] - gu[l]);
    gvd[l] = zsdotp[l] * (gv[l + 1] - gv[l]);
  }
  // Level tendencies go out as soon as they are formed (fewer live arrays).
  zsumd = zvgpg[0] * ds[0];
  const float rdsig0 = rd[0];
  F.gp[c] = ps;
  F.gtn[c] = gt[0] * gd[0] - K.AKAP * ztv2[0] * gd[0] - rdsig0 * (gtd[0] + t01[0] * (sh[0] * gvp - zsumd));
  F.gqn[c] = -rdsig0 * gqm[0];
  F.guz[c] = -gu[0] * gz[0] - gpj * ztv1[0] - rdsig0 * gvd[0];
  F.gvz[c] = gv[0] * gz[0] - gpm * ztv1[0] - rdsig0 * gud[0];
  F.dw[c] = gd[0] * ps * K.PSURF * K.WW;
#pragma unroll
  for (int l = 1; l < NL; ++l) {
    const int column = l * NL;
    float ztpta = C[column] * zvgpg[0];
    float ztptb = C[column] * (zvgpg[0] + gd[0]);
#pragma unroll
    for (int j = 1; j <= l; ++j) {
      ztpta = ztpta + C[column + j] * zvgpg[j];
      ztptb = ztptb + C[column + j] * (zvgpg[j] + gd[j]);
    }
    const float rdsig = rd[l], t01s2 = t01[l], t01s2m = t01[l - 1], sigmah = sh[l], sigmahm = sh[l - 1];
    const float tkp = tkpT[l];
    const size_t at = l * SN + c;
    if (l < NL - 1) {
      zsumd = zsumd + zvgpg[l] * ds[l];
      F.gtn[at] = gt[l] * gd[l] + K.AKAP * ztv2[l] * (zvgpg[l] - ztptb) + tkp * (zvgpg[l] - ztpta) -
               rdsig * (gtd[l] + gtd[l - 1] + gvp * (t01s2 * sigmah + t01s2m * sigmahm) - zsumd * (t01s2m + t01s2) +
                        zvgpg[l] * ds[l] * t01s2m);
      F.gqn[at] = -rdsig * (gqm[l] - gqm[l - 1]);
      F.guz[at] = -gu[l] * gz[l] - gpj * ztv1[l] - rdsig * (gvd[l] + gvd[l - 1]);
      F.gvz[at] = gv[l] * gz[l] - gpm * ztv1[l] - rdsig * (gud[l] + gud[l - 1]);
    } else {
      F.gtn[at] = gt[l] * gd[l] + K.AKAP * ztv2[l] * (zvgpg[l] - ztptb) + tkp * (zvgpg[l] - ztpta) -
               rdsig * (gtd[NL - 2] + t01s2m * (sigmahm * gvp - zsumd));
      F.gqn[at] = rdsig * gqm[NL - 2];
      F.guz[at] = -gu[l] * gz[l] - gpj * ztv1[l] - rdsig * gvd[NL - 2];
      F.gvz[at] = gv[l] * gz[l] - gpm * ztv1[l] - rdsig * gud[NL - 2];
    }
    F.dw[at] = (zvgpg[l] - ztptb) * ps * K.PSURF * K.WW;
  }
  const float scale = sqrtf(rcsq);
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    float gsum = 0.f;
#pragma unroll
    for (int k = 0; k < NL; ++k) gsum = gsum + G[l * NL + k] * (ztv1[k] - gt[k]);
    const float gphi = gsum * 2.f / rcsq;
    const size_t at = l * SN + c;
    F.gut[at] = gu[l] * gt[l];
    F.gvt[at] = gv[l] * gt[l];
    F.gke[at] = gu[l] * gu[l] + gv[l] * gv[l] + gphi;
    F.guq[at] = gu[l] * gq[l];
    F.gvq[at] = gv[l] * gq[l];
    F.du0[at] = K.CV * gu[l] * scale;
    F.dv0[at] = K.CV * gv[l] * scale;
  }
  F.gvpp[c] = gvp;
  F.dp0[c] = K.PSURF * ps;
}

// spectrala for one real spectral coefficient (dynamics/wgsl/spectrala.wgsl):
// the Hoskins-Simmons semi-implicit scheme with this slot's bm1 for its phase.
// At least three resident blocks per SM: with its last pass read ahead, the
// registers that a looser bound allows measured faster than five blocks.
template <int NL>
__global__ void __launch_bounds__(kBlock, 3) k_spectrala(Model m) {
  const Dims& d = m.d;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.S * d.NRSP) return;
  const int slot = c / d.NRSP, s = c % d.NRSP;
  const StepParams& P = m.params[slot];
  if (!P.active) return;
  const PlanetConst& K = m.pc[slot];
  const float* tb = slot_tabs(m, slot);
  const float* G = tb + m.to.g;
  const float* t0T = tb + m.to.t0;
  const float* ds = tb + m.to.dsigma;
  const float* tau = tb + m.to.tau;
  const float* bm1 = tb + m.to.bm1 + (size_t)P.phase * d.T * NL * NL;
  const size_t SR = (size_t)d.S * d.NRSP;
  const FieldPtrs& F = m.f;
  const bool filter = P.filter != 0.f;
  const float DELT = P.delt, DELT2 = P.delt2;
  const float apm = F.spm[c];
  float adm[NL], azm[NL], atm[NL], aqm[NL], adt[NL], stt[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SR + c;
    adm[l] = F.sdm[at];
    azm[l] = F.szm[at];
    atm[l] = F.stm[at];
    aqm[l] = F.sqm[at];
    adt[l] = F.sdt[at];
    stt[l] = F.stt[at];
  }
  float zgt[NL], zgm[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    float gt = 0.f, gm = 0.f;
#pragma unroll
    for (int k = 0; k < NL; ++k) {
      gt = gt + G[l * NL + k] * stt[k];
      gm = gm + G[l * NL + k] * atm[k];
    }
    zgt[l] = gt;
    zgm[l] = gm;
  }
  float spt = F.spt[c];
  const float spm = apm;
  const float sop = tb[m.to.sop + s];
  const int jn = (int)m.sh.nindex[s];
  float sdt[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    float zsum = 0.f;
    if (jn > 0) {
      const float zq = 1.f / (float)(jn * (jn + 1));
#pragma unroll
      for (int l2 = 0; l2 < NL; ++l2) {
        const float z0 = t0T[l2];
        const float zt = zgt[l2] - z0 * spt;
        const float zm = zgm[l2] + z0 * spm;
        const float za = adt[l2] * zq + sop;
        const float zb = adm[l2] * zq;
        const float zz = zb + DELT * (zm + za + DELT * zt);
        zsum = zsum + zz * bm1[((jn - 1) * NL + l) * NL + l2];
      }
    }
    sdt[l] = s < 2 ? 0.f : zsum;
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) spt = spt + ds[l] * sdt[l];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < NL; ++k) t = t + tau[l * NL + k] * sdt[k];
    stt[l] = stt[l] - t;
  }
  const float spp = F.spp[c];
  if (filter) F.spm[c] = K.PNU21 * spp + K.PNU * apm;
  const float sppNew = s < 2 ? 0.f : apm - DELT2 * spt;
  F.spp[c] = sppNew;
  F.sp[c] = sppNew;
  F.spt[c] = spt;
  // The last pass runs in two halves of levels, each reading all its inputs
  // before its stores: the fields are distinct arrays, but the compiler
  // cannot prove it and would otherwise wait for each level's loads in turn.
  constexpr int H = (NL + 1) / 2;
  const float PNU21 = K.PNU21, PNU = K.PNU;
#pragma unroll
  for (int h0 = 0; h0 < NL; h0 += H) {
    float szt_[H], sqt_[H], sdp_[H], szp_[H], stp_[H], sqp_[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
      const int l = h0 + i;
      if (l >= NL) break;
      const size_t at = l * SR + c;
      szt_[i] = F.szt[at];
      sqt_[i] = F.sqt[at];
      if (filter) {
        sdp_[i] = F.sdp[at];
        szp_[i] = F.szp[at];
        stp_[i] = F.stp[at];
        sqp_[i] = F.sqp[at];
      }
    }
#pragma unroll
    for (int i = 0; i < H; ++i) {
      const int l = h0 + i;
      if (l >= NL) break;
      const size_t at = l * SR + c;
      if (filter) {
        F.sdm[at] = PNU21 * sdp_[i] + PNU * adm[l];
        F.szm[at] = PNU21 * szp_[i] + PNU * azm[l];
        F.stm[at] = PNU21 * stp_[i] + PNU * atm[l];
        F.sqm[at] = PNU21 * sqp_[i] + PNU * aqm[l];
      }
      const float sdp = 2.f * sdt[l] - adm[l];
      const float stp = DELT2 * stt[l] + atm[l];
      const float szp = DELT2 * szt_[i] + azm[l];
      const float sqp = DELT2 * sqt_[i] + aqm[l];
      F.sdt[at] = sdt[l];
      F.stt[at] = stt[l];
      F.sdp[at] = sdp;
      F.stp[at] = stp;
      F.szp[at] = szp;
      F.sqp[at] = sqp;
      F.sd[at] = sdp;
      F.st[at] = stp;
      F.sz[at] = szp;
      F.sq[at] = sqp;
    }
  }
}

__device__ __forceinline__ float2 ld2(const float* p, size_t i) { return *reinterpret_cast<const float2*>(p + i); }
__device__ __forceinline__ void st2(float* p, size_t i, float2 v) { *reinterpret_cast<float2*>(p + i) = v; }

// spectrald up to mkdheat (dynamics/wgsl/spectrald-diffusion.wgsl). A thread
// owns two adjacent real coefficients (NRSP is even, so both are of one
// slot) of one level. Every input is read before the slot's parameters are
// tested and before the first store: the fields are distinct arrays, but
// the compiler cannot prove it, and would otherwise order each load after
// the stores before it.
__global__ void __launch_bounds__(kBlock) k_spectrald_diffusion(Model m) {
  const Dims& d = m.d;
  const int c = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (c >= d.S * d.NRSP) return;
  const int l = blockIdx.y;
  const int slot = c / d.NRSP, s = c - slot * d.NRSP;
  const float* tb = slot_tabs(m, slot);
  const size_t at = (size_t)l * d.S * d.NRSP + c;
  const FieldPtrs& F = m.f;
  const float2 szp0 = ld2(F.szp, at), szt0 = ld2(F.szt, at), stp0 = ld2(F.stp, at), stt0 = ld2(F.stt, at);
  const float2 sdp0 = ld2(F.sdp, at), sdt0 = ld2(F.sdt, at), sqp0 = ld2(F.sqp, at), sqt0 = ld2(F.sqt, at);
  const float* sak = tb + m.to.sakpp + l * d.NRSP + s;
  const float* srpl = tb + m.to.srp + l * d.NRSP + s;
  const float sakpp[2] = {sak[0], sak[1]}, srp[2] = {srpl[0], srpl[1]};
  const float damp = tb[m.to.damp + l], tdisst = tb[m.to.tdisst + l], tdissq = tb[m.to.tdissq + l];
  const float tdissd = tb[m.to.tdissd + l], tdissz = tb[m.to.tdissz + l], tfrc = tb[m.to.tfrc + l];
  const StepParams& P = m.params[slot];
  if (!P.active) return;
  const float D2 = P.delt2, PLAVOR = m.pc[slot].PLAVOR;
  float o[12][2];  // szp, stp, sdp, sqp, stt, sqt, sdt, szt, zdsdp1, zdszp1, zdsdp2, zdszp2
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const float szp = (k ? szp0.y : szp0.x) + D2 * (k ? szt0.y : szt0.x);
    const float stp = (k ? stp0.y : stp0.x) + D2 * (k ? stt0.y : stt0.x);
    const float sdp = (k ? sdp0.y : sdp0.x) + D2 * (k ? sdt0.y : sdt0.x);
    const float sqp = (k ? sqp0.y : sqp0.x) + D2 * (k ? sqt0.y : sqt0.x);
    // IEEE divisions (the file otherwise divides to 2 ulp): the diffusion
    // and friction increments feed mkdheat's heating through two more
    // transforms, where 2-ulp quotients left V3's bound.
    const float sk = sakpp[k];
    const float stt = __fdiv_rn((-damp - tdisst * sk) * stp + damp * srp[k], 1.f + D2 * (damp + tdisst * sk));
    const float sqt = __fdiv_rn(-tdissq * sk * sqp, 1.f + D2 * tdissq * sk);
    const float zsdt1 = __fdiv_rn(-tfrc * sdp, 1.f + D2 * tfrc);
    const float zsdt2 = __fdiv_rn(-tdissd * sk * sdp, 1.f + D2 * tdissd * sk);
    float zszt1 = __fdiv_rn(-tfrc * szp, 1.f + D2 * tfrc);
    float zszt2 = __fdiv_rn(-tdissz * sk * szp, 1.f + D2 * tdissz * sk);
    float szt = zszt1 + zszt2;
    if (s + k == 2) {
      zszt1 = zszt1 + __fdiv_rn(PLAVOR * tfrc, 1.f + D2 * tfrc);
      zszt2 = zszt2 + __fdiv_rn(PLAVOR * tdissz * sk, 1.f + D2 * tdissz * sk);
      szt = szt + PLAVOR * (__fdiv_rn(tfrc, 1.f + D2 * tfrc) + __fdiv_rn(tdissz * sk, 1.f + D2 * tdissz * sk));
    }
    const float v[12] = {szp, stp, sdp, sqp, stt, sqt, zsdt1 + zsdt2, szt, zsdt1 * D2, zszt1 * D2, zsdt2 * D2,
                         zszt2 * D2};
#pragma unroll
    for (int j = 0; j < 12; ++j) o[j][k] = v[j];
  }
  if (l == 0 && s < 2) st2(F.spp, c, make_float2(0.f, 0.f));
  float* const dst[12] = {F.szp, F.stp, F.sdp, F.sqp, F.stt, F.sqt, F.sdt, F.szt, F.zdsdp1, F.zdszp1, F.zdsdp2, F.zdszp2};
#pragma unroll
  for (int j = 0; j < 12; ++j) st2(dst[j], at, make_float2(o[j][0], o[j][1]));
}

// Elementwise grid-point kernels give each thread four adjacent columns of
// one level (16-byte loads and stores): a block covers kCols4 = 512
// columns, and 512 divides NHOR (2048, 8192, 18432), so a block's columns
// share one slot. Four columns per thread keep four times the bytes in
// flight for the same number of resident warps.
constexpr int kCols4 = 4 * kBlock;

__device__ __forceinline__ float4 ld4(const float* p, size_t i) { return *reinterpret_cast<const float4*>(p + i); }
__device__ __forceinline__ void st4(float* p, size_t i, float4 v) { *reinterpret_cast<float4*>(p + i) = v; }

// mkdheat's grid-point stages (dynamics/wgsl/mkdheat.wgsl).
__global__ void __launch_bounds__(kBlock) k_mkdheat(Model m, int stage) {
  const Dims& d = m.d;
  const int slot = blockIdx.x * kCols4 / d.NHOR;
  const int c = blockIdx.x * kCols4 + 4 * threadIdx.x;
  const int l = blockIdx.y;
  const size_t i = (size_t)l * d.S * d.NHOR + c;
  const int h = c - slot * d.NHOR;
  const FieldPtrs& F = m.f;
  // inputs first, then the slot's parameters
  const float4 dq = ld4(F.dq, i);
  const float4 dp = stage == 1 ? make_float4(0.f, 0.f, 0.f, 0.f) : ld4(F.dp, c);
  const float4 ek = stage == 3 ? ld4(F.zdekin, i) : make_float4(0.f, 0.f, 0.f, 0.f);
  float4 zu = ek, zv = ek, zdu = ek, zdv = ek, rc = ek;
  if (stage != 3) {
    zu = ld4(F.zu, i);
    zv = ld4(F.zv, i);
    zdu = ld4(F.zdu, i);
    zdv = ld4(F.zdv, i);
    rc = ld4(m.sh.rcsq, h);
  }
  const float ds = m.tabs[(size_t)slot * m.to.stride + m.to.dsigma + l];
  const StepParams& P = m.params[slot];
  if (!P.active) return;
  const PlanetConst& K = m.pc[slot];
  const float4 heat = make_float4(1.f + K.ADV * dq.x, 1.f + K.ADV * dq.y, 1.f + K.ADV * dq.z, 1.f + K.ADV * dq.w);
  if (stage == 3) {
    // IEEE divisions throughout mkdheat, as in spectrald's diffusion.
    auto one = [&](float e, float ht, float p) {
      const float dtdt = __fdiv_rn(__fdiv_rn(__fdiv_rn(__fdiv_rn(-e * 0.5f, K.ACPD), ht), p) * K.GA, ds);
      return __fdiv_rn(__fdiv_rn(dtdt, K.CT), K.WW);
    };
    st4(F.zdtdt, i, make_float4(one(ek.x, heat.x, dp.x), one(ek.y, heat.y, dp.y), one(ek.z, heat.z, dp.z),
                                one(ek.w, heat.w, dp.w)));
    return;
  }
  auto one = [&](float r, float zu1, float zv1, float zdu1, float zdv1, float ht, float p) {
    const float scale = K.CV * sqrtf(r);
    const float u = zu1 * scale, v = zv1 * scale, du = zdu1 * scale, dv = zdv1 * scale;
    const float change = du * (2.f * u + du) + dv * (2.f * v + dv);
    if (stage == 1) {
      const float dtdt = __fdiv_rn(__fdiv_rn(__fdiv_rn(-change, P.deltsec2) * 0.5f, K.ACPD), ht);
      return __fdiv_rn(__fdiv_rn(dtdt, K.CT), K.WW);
    }
    return __fdiv_rn(__fdiv_rn(change, P.deltsec2) * p, K.GA) * ds;
  };
  const float4 r = make_float4(one(rc.x, zu.x, zv.x, zdu.x, zdv.x, heat.x, dp.x),
                               one(rc.y, zu.y, zv.y, zdu.y, zdv.y, heat.y, dp.y),
                               one(rc.z, zu.z, zv.z, zdu.z, zdv.z, heat.z, dp.z),
                               one(rc.w, zu.w, zv.w, zdu.w, zdv.w, heat.w, dp.w));
  st4(stage == 1 ? F.zdtdt : F.zdekin, i, r);
}

// mkdheat's zsdef(2:NESP,:) = 0 (dynamics/wgsl/mean-mode.wgsl).
// One block row per plane: blockIdx.y = slot, blockIdx.z = level.
__global__ void k_mean_mode(float* t, int nrsp) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrsp || r == 0) return;
  t[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * nrsp + r] = 0.f;
}

// spectrald after mkdheat (dynamics/wgsl/spectrald-update.wgsl), two
// adjacent real coefficients of one level per thread, inputs read first.
__global__ void __launch_bounds__(kBlock) k_spectrald_update(Model m) {
  const Dims& d = m.d;
  const int c = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (c >= d.S * d.NRSP) return;
  const int l = blockIdx.y;
  const int slot = c / d.NRSP;
  const size_t at = (size_t)l * d.S * d.NRSP + c;
  const FieldPtrs& F = m.f;
  const float2 stt0 = ld2(F.stt, at), zstt1 = ld2(F.zstt1, at), zstt2 = ld2(F.zstt2, at);
  const float2 szp0 = ld2(F.szp, at), szt = ld2(F.szt, at), stp0 = ld2(F.stp, at), sdp0 = ld2(F.sdp, at);
  const float2 sdt = ld2(F.sdt, at), sqp0 = ld2(F.sqp, at), sqt = ld2(F.sqt, at);
  const bool surface = l == 0;  // the level-0 threads also update sp
  const float2 spp = surface ? ld2(F.spp, c) : make_float2(0.f, 0.f);
  const StepParams& P = m.params[slot];
  if (!P.active) return;
  const float PNU = m.pc[slot].PNU;
  const bool filter = P.filter != 0.f;
  const float D2 = P.delt2;
  float2 szm = make_float2(0.f, 0.f), stm = szm, sdm = szm, sqm = szm, spm = szm;
  if (filter) {
    szm = ld2(F.szm, at);
    stm = ld2(F.stm, at);
    sdm = ld2(F.sdm, at);
    sqm = ld2(F.sqm, at);
    if (surface) spm = ld2(F.spm, c);
  }
  const float2 stt = make_float2(stt0.x + zstt1.x + zstt2.x, stt0.y + zstt1.y + zstt2.y);
  const float2 szp = make_float2(szp0.x + D2 * szt.x, szp0.y + D2 * szt.y);
  const float2 stp = make_float2(stp0.x + D2 * stt.x, stp0.y + D2 * stt.y);
  const float2 sdp = make_float2(sdp0.x + D2 * sdt.x, sdp0.y + D2 * sdt.y);
  const float2 sqp = make_float2(sqp0.x + D2 * sqt.x, sqp0.y + D2 * sqt.y);
  if (surface) {
    if (filter) st2(F.spm, c, make_float2(spm.x + PNU * spp.x, spm.y + PNU * spp.y));
    st2(F.sp, c, spp);
  }
  st2(F.stt, at, stt);
  st2(F.szp, at, szp);
  st2(F.stp, at, stp);
  st2(F.sdp, at, sdp);
  st2(F.sqp, at, sqp);
  if (filter) {
    st2(F.szm, at, make_float2(szm.x + PNU * szp.x, szm.y + PNU * szp.y));
    st2(F.stm, at, make_float2(stm.x + PNU * stp.x, stm.y + PNU * stp.y));
    st2(F.sdm, at, make_float2(sdm.x + PNU * sdp.x, sdm.y + PNU * sdp.y));
    st2(F.sqm, at, make_float2(sqm.x + PNU * sqp.x, sqm.y + PNU * sqp.y));
  }
  st2(F.sz, at, szp);
  st2(F.st, at, stp);
  st2(F.sd, at, sdp);
  st2(F.sq, at, sqp);
}

// gridpointd before the parameterizations (dynamics/wgsl/physics-in.wgsl),
// one thread per column, every input read before the first store. A block's
// columns share one slot: kBlock divides NHOR. The grid tendencies, and the
// dimensional ones below the surface level, are zeroed only under
// single-stage replay (Model::zero_gdt).
template <int NL>
__global__ void __launch_bounds__(kBlock) k_physics_in(Model m) {
  const Dims& d = m.d;
  const int slot = blockIdx.x * kBlock / d.NHOR;
  if (!m.params[slot].active) return;
  const int c = blockIdx.x * kBlock + threadIdx.x;
  const int h = c - slot * d.NHOR;
  const PlanetConst& K = m.pc[slot];
  const float PSURF = K.PSURF, CV = K.CV, CT = K.CT;
  const float* t0 = m.tabs + (size_t)slot * m.to.stride + m.to.t0;
  const size_t SN = (size_t)d.S * d.NHOR;
  const FieldPtrs& F = m.f;
  const float gp = F.gp[c], rcsq = m.sh.rcsq[h];
  float gu[NL], gv[NL], gt[NL], gq[NL], t0l[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    gu[l] = F.gu[at];
    gv[l] = F.gv[at];
    gt[l] = F.gt[at];
    gq[l] = F.gq[at];
    t0l[l] = t0[l];
  }
  const float dp = PSURF * expf(gp);
  F.dp[c] = dp;
  const float scale = sqrtf(rcsq);
#pragma unroll
  for (int l = 0; l < NL + 1; ++l) {
    const size_t at = l * SN + c;
    if (m.zero_gdt || l == NL) {
      F.dudt[at] = 0.f;
      F.dvdt[at] = 0.f;
      F.dtdt[at] = 0.f;
      F.dqdt[at] = 0.f;
    }
    if (l < NL) {
      if (m.zero_gdt) {
        F.gudt[at] = 0.f;
        F.gvdt[at] = 0.f;
        F.gtdt[at] = 0.f;
        F.gqdt[at] = 0.f;
      }
      F.du[at] = CV * gu[l] * scale;
      F.dv[at] = CV * gv[l] * scale;
      F.dt[at] = CT * (gt[l] + t0l[l]);
      F.dq[at] = gq[l] * PSURF / dp;
    }
  }
}

// gridpointd after the parameterizations (dynamics/wgsl/physics-out.wgsl),
// four columns of one level per thread, inputs read before the stores.
// Within a full step gudt, gvdt, gtdt hold no earlier increment and are not
// read (Model::zero_gdt): the sum adds +0 as the zeroed fields would.
__global__ void __launch_bounds__(kBlock) k_physics_out(Model m) {
  const Dims& d = m.d;
  const int slot = blockIdx.x * kCols4 / d.NHOR;
  const int c = blockIdx.x * kCols4 + 4 * threadIdx.x;
  const int h = c - slot * d.NHOR;
  const size_t i = (size_t)blockIdx.y * d.S * d.NHOR + c;
  const FieldPtrs& F = m.f;
  const float4 dudt = ld4(F.dudt, i), dvdt = ld4(F.dvdt, i), dtdt = ld4(F.dtdt, i), dqdt = ld4(F.dqdt, i);
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  const bool earlier = m.zero_gdt != 0;
  const float4 gudt = earlier ? ld4(F.gudt, i) : z, gvdt = earlier ? ld4(F.gvdt, i) : z;
  const float4 gtdt = earlier ? ld4(F.gtdt, i) : z, gqdt = ld4(F.gqdt, i);
  const float4 dp = ld4(F.dp, c), rc = ld4(m.sh.rcsq, h);
  if (!m.params[slot].active) return;
  const PlanetConst& K = m.pc[slot];
  const float CV = K.CV, WW = K.WW, CT = K.CT, PSURF = K.PSURF;
  const float4 scale = make_float4(sqrtf(rc.x), sqrtf(rc.y), sqrtf(rc.z), sqrtf(rc.w));
  auto wind = [&](float4 t, float4 g) {
    return make_float4(t.x / scale.x / CV / WW + g.x, t.y / scale.y / CV / WW + g.y, t.z / scale.z / CV / WW + g.z,
                       t.w / scale.w / CV / WW + g.w);
  };
  st4(F.gudt, i, wind(dudt, gudt));
  st4(F.gvdt, i, wind(dvdt, gvdt));
  st4(F.gtdt, i, make_float4(dtdt.x / CT / WW + gtdt.x, dtdt.y / CT / WW + gtdt.y, dtdt.z / CT / WW + gtdt.z,
                             dtdt.w / CT / WW + gtdt.w));
  st4(F.gqdt, i, make_float4(dqdt.x * dp.x / WW / PSURF + gqdt.x, dqdt.y * dp.y / WW / PSURF + gqdt.y,
                             dqdt.z * dp.z / WW / PSURF + gqdt.z, dqdt.w * dp.w / WW / PSURF + gqdt.w));
}

inline unsigned blocks(size_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

void dyn_calcgp(const Model& m, cudaStream_t st) {
  static_assert(2048 % kBlock == 0, "k_calcgp assumes a block lies in one slot");
  const unsigned n = (unsigned)((size_t)m.d.S * m.d.NHOR / kBlock);
  if (m.d.L == 10)
    k_calcgp<10><<<n, kBlock, 0, st>>>(m);
  else
    k_calcgp<5><<<n, kBlock, 0, st>>>(m);
}
void dyn_spectrala(const Model& m, cudaStream_t st) {
  const unsigned n = blocks((size_t)m.d.S * m.d.NRSP, kBlock);
  if (m.d.L == 10)
    k_spectrala<10><<<n, kBlock, 0, st>>>(m);
  else
    k_spectrala<5><<<n, kBlock, 0, st>>>(m);
}
void dyn_spectrald_diffusion(const Model& m, cudaStream_t st) {
  const dim3 grid(blocks((size_t)m.d.S * m.d.NRSP / 2, kBlock), m.d.NLEV);
  k_spectrald_diffusion<<<grid, kBlock, 0, st>>>(m);
}
void dyn_mkdheat(const Model& m, int stage, cudaStream_t st) {
  const dim3 grid((unsigned)((size_t)m.d.S * m.d.NHOR / kCols4), m.d.NLEV);
  k_mkdheat<<<grid, kBlock, 0, st>>>(m, stage);
}
void dyn_mean_mode(const Model& m, float* target, cudaStream_t st) {
  const dim3 grid(blocks((size_t)m.d.NRSP, 256), m.d.S, m.d.NLEV);
  k_mean_mode<<<grid, 256, 0, st>>>(target, m.d.NRSP);
}
void dyn_spectrald_update(const Model& m, cudaStream_t st) {
  const dim3 grid(blocks((size_t)m.d.S * m.d.NRSP / 2, kBlock), m.d.NLEV);
  k_spectrald_update<<<grid, kBlock, 0, st>>>(m);
}
void dyn_physics_in(const Model& m, cudaStream_t st) {
  const unsigned n = (unsigned)((size_t)m.d.S * m.d.NHOR / kBlock);
  if (m.d.L == 10)
    k_physics_in<10><<<n, kBlock, 0, st>>>(m);
  else
    k_physics_in<5><<<n, kBlock, 0, st>>>(m);
}
void dyn_physics_out(const Model& m, cudaStream_t st) {
  const dim3 grid((unsigned)((size_t)m.d.S * m.d.NHOR / kCols4), m.d.NLEV);
  k_physics_out<<<grid, kBlock, 0, st>>>(m);
}

}  // namespace exogcm
