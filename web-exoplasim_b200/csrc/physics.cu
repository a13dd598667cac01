// Column physics of the GCM step for every slot of a batch (FP32), plus the
// per-planet reductions and the snapshot pack.
//
// Arithmetic follows src/model/climate/gcm/physics/*/wgsl/*.wgsl and
// snapshot/wgsl/pack.wgsl (ExoPlaSim's miscmod fixer, fluxmod, radmod,
// rainmod, landmod, vegmod, glaciermod, icemod, oceanmod, seamod,
// carbonmod). One thread owns one column c = slot * NHOR + h of the batch and
// keeps its levels in registers (kernels are instantiated per level count).
// The reference's per-planet global sums (fixer, getiflx) and the mkdca pass
// limit run as one block per slot with a fixed summation order, in FP64.
// The fixer's apply step, the surface fluxes, vertical diffusion, solar
// angle and ozone are in physics_flux.cu (IEEE division).
#include "physics_common.cuh"

namespace exogcm {

namespace {

// ---------------------------------------------------------------- fixer
// physics/fixer/wgsl/column.wgsl: fix0d per column.
template <int NL>
__global__ void __launch_bounds__(kBlock) k_fixer_column(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const float* ds = tb + m.to.dsigma;
  // dq stays in registers for the stores below (a reload after each store
  // would wait for it: the compiler cannot prove the fields distinct)
  float dq[NL], negative = 0.f, positive = 0.f;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    dq[l] = F.dq[l * SN + c];
    const float q = dq[l] * ds[l];
    if (dq[l] < 0.f) negative = negative + q;
    if (dq[l] > 0.f) positive = positive + q;
  }
  const float zgw = m.sh.zgw[h];
  float zneg = -negative * F.dp[c] * zgw;
  float zpos = positive * F.dp[c] * zgw;
  float factor = 1.f;
  const bool fixed = zneg > 0.f && zpos >= zneg;
  if (fixed) {
    factor = (zpos - zneg) / zpos;
    zneg = 0.f;
    zpos = zpos * factor;
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) F.fixq[l * SN + c] = fixed ? fmaxf(dq[l] * factor, 0.f) : dq[l];
  F.fixneg[c] = zneg;
  F.fixpos[c] = zpos;
}

// physics/fixer/wgsl/row.wgsl: fix1d per latitude row, summed in longitude
// order. One warp per row: its lanes stage the row in shared memory with
// coalesced loads, lane 0 adds the values in longitude order (the shader's
// sums, bit for bit), and the update of a fixed row runs over all lanes.
constexpr int kRowWarps = 4;
constexpr int kMaxNlon = 192;  // NLON at T63, the largest truncation an engine accepts

template <int NL>
__global__ void __launch_bounds__(32 * kRowWarps) k_fixer_row(Model m) {
  __shared__ float stage[kRowWarps][kMaxNlon];
  const Dims& d = m.d;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * kRowWarps + warp;
  if (r >= d.S * d.NLAT) return;  // the whole warp
  const int slot = r / d.NLAT;
  if (!m.params[slot].active) return;
  const size_t SN = (size_t)d.S * d.NHOR;
  const FieldPtrs& F = m.f;
  const int first = r * d.NLON;  // slot * NHOR + lat * NLON
  float* row = stage[warp];
  auto ordered_sum = [&](const float* src) {
    for (int j = lane; j < d.NLON; j += 32) row[j] = src[first + j];
    __syncwarp();
    float sum = 0.f;
    if (lane == 0)
      for (int j = 0; j < d.NLON; ++j) sum = sum + row[j];
    sum = __shfl_sync(0xffffffffu, sum, 0);
    __syncwarp();  // the row buffer is staged again next
    return sum;
  };
  const float zneg = ordered_sum(F.fixneg);
  if (zneg <= 0.f) return;
  const float zpos = ordered_sum(F.fixpos);
  if (zpos < zneg) return;
  const float factor = (zpos - zneg) / zpos;
  for (int j = lane; j < d.NLON; j += 32) {
    float q[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) q[l] = F.fixq[l * SN + first + j];
    const float pos = F.fixpos[first + j];
#pragma unroll
    for (int l = 0; l < NL; ++l) F.fixq[l * SN + first + j] = fmaxf(q[l] * factor, 0.f);
    F.fixneg[first + j] = 0.f;
    F.fixpos[first + j] = pos * factor;
  }
}

// Per-slot global sums of two grid fields in FP64 with a fixed order (the
// reference's reduction/wgsl/sum.wgsl, kept in double as the build asks of
// global budget reductions). Writes the sums as floats to target[0|1 * S + slot]
// and as doubles to sums[slot * 4 + which * 2 + 0|1].
__global__ void __launch_bounds__(kSumThreads) k_slot_sums(Model m, const float* a, const float* b, float* target,
                                                           int which) {
  const Dims& d = m.d;
  const int slot = blockIdx.x;
  if (!m.params[slot].active) return;
  if (which == 1 && m.params[slot].coupled == 0.f) return;  // getiflx runs with icestep only
  __shared__ double sa[kSumThreads], sb[kSumThreads];
  double x = 0.0, y = 0.0;
  const size_t base = (size_t)slot * d.NHOR;
  for (int h = threadIdx.x; h < d.NHOR; h += kSumThreads) {
    x += (double)a[base + h];
    y += (double)b[base + h];
  }
  sa[threadIdx.x] = x;
  sb[threadIdx.x] = y;
  __syncthreads();
  for (int stride = kSumThreads / 2; stride > 0; stride /= 2) {
    if (threadIdx.x < stride) {
      sa[threadIdx.x] += sa[threadIdx.x + stride];
      sb[threadIdx.x] += sb[threadIdx.x + stride];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    target[slot] = (float)sa[0];
    target[d.S + slot] = (float)sb[0];
    m.sums[slot * 4 + which * 2] = sa[0];
    m.sums[slot * 4 + which * 2 + 1] = sb[0];
  }
}

// ---------------------------------------------------------------- radiation
__device__ __forceinline__ float ozone_absorption(float o3, float zsolar1) {
  return (0.02118f * o3 / (1.f + 0.042f * o3 + 0.000323f * (o3 * o3)) + 1.082f * o3 / fpow(1.f + 138.6f * o3, 0.805f) +
          0.0658f * o3 / (1.f + (103.6f * o3) * (103.6f * o3) * (103.6f * o3))) /
         zsolar1;
}
__device__ __forceinline__ float vapour_absorption(float wv, float zsolar2) {
  return 2.9f * wv / (fpow(1.f + 141.5f * wv, 0.635f) + 5.925f * wv) / zsolar2;
}

// Per-level state of one swr band for the block's threads, [level][thread]
// in shared memory: the level loops stay rolled, so both bands' code fits
// the instruction cache, and the accesses are conflict-free.
struct SwrLevels {
  float* p;
  __device__ float& at(int array, int level) const { return p[(array * (MAXLEV + 1) + level) * kBlock + threadIdx.x]; }
  static constexpr int MAXLEV = 10;
  static constexpr int kArrays = 6;  // tl, rls (NL + 1 levels), tbd, tbu, rb, rbs
};

// One band of swr (physics/radiation/wgsl/swr.wgsl) for one column: ozone
// absorption below 0.75 um (BAND 0) or water vapour above (BAND 1), by the
// adding method. The band's cloud optics, layer reflectances and
// transmissivities follow the shader's expressions in its order; the flux
// of each level goes to fu/fd (shared memory, [level][column]) as soon as
// the upward pass reaches it. Returns the new surface albedos (nalb1,
// nalb2, albedo) the column writes.
template <int NL, int BAND>
__device__ __forceinline__ void swr_band(const Model& m, const PlanetConst& K, const float* tb, size_t SN, int c,
                                         float mu0, float ftop, SwrLevels lv, float* fu, float* fd, int stride,
                                         float* alb) {
  enum { TL = 0, RLS = 1, TBD = 2, TBU = 3, RB = 4, RBS = 5 };
  const FieldPtrs& F = m.f;
  const float ZBETTA = 1.66f, ZMBAR = 1.9f, ZFO3 = 100.f / 2.14f, ZMU00 = 0.5f, INV_LN10 = 0.43429448190325176f;
  const float diffusivity = BAND == 0 ? ZMBAR : ZBETTA;
  const float* ds = tb + m.to.dsigma;
  const float* sg = tb + m.to.sigma;
  const float dp = F.dp[c];
  const float zm = 35.f / sqrtf(1.f + 1224.f * mu0 * mu0);
  // The absorber amount of level l from its loaded inputs (BAND 0: ozone;
  // BAND 1: water vapour q and temperature t).
  auto amount_of = [&](float dsigma, float q, float t, float sgl) {
    return BAND == 0 ? ZFO3 * dsigma * dp * q / K.GA
                     : 0.1f * dsigma * q * dp / K.GA * sqrtf(273.f / t) * sgl * dp / 100000.f;
  };
  auto absorber = [&](int l) { return BAND == 0 ? F.dqo3[l * SN + c] : F.dq[l * SN + c]; };
  auto amount_at = [&](int l) { return amount_of(ds[l], absorber(l), BAND == 0 ? 0.f : F.dt[l * SN + c], sg[l]); };
  auto absorption = [&](float x) {
    return BAND == 0 ? ozone_absorption(x, K.ZSOLAR1) : vapour_absorption(x, K.ZSOLAR2);
  };
  // The downward pass reads each level's cloud water one level ahead; the
  // column totals below read every other input, so only that one is
  // fetched into L2 here.
#pragma unroll
  for (int l = 0; l < NL; ++l) prefetch_l2(F.dql + l * SN + c);
  // Column totals of the absorber path (slant above the first cloud,
  // diffuse below).
  float pt = 0.f, xpt = 0.f, cs = 1.f;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const float amount = amount_at(l);
    pt = pt + amount;
    xpt = cs * (xpt + zm * amount) + (1.f - cs) * (xpt + diffusivity * amount);
    cs = cs * (1.f - F.dcc[l * SN + c]);
  }
  const float ccn = F.dcc[(NL - 1) * SN + c];
  float rcsSurface = 0.f, rcsuSurface = 0.f;
  if (BAND == 0) {
    const float scf = K.RCOEFF * dp / 101100.f * 9.80665f / K.GA;
    const float diffuseRayleigh = 1.f - expf(scf * K.LN_DIFFUSE_RAYLEIGH);
    rcsuSurface = diffuseRayleigh * (1.f - ccn);
    rcsSurface =
        (1.f - expf(scf * logf(1.f - 0.219f / (1.f + 0.816f * mu0)))) * cs + diffuseRayleigh * (1.f - cs - ccn);
  }
  // Downward pass: layer properties and the adding recursion from the top.
  float ta = 1.f, tas = 1.f, ra = 0.f, ras = 0.f;
  float tt = 1.f, ttu = 1.f - absorption(xpt + diffusivity * pt);
  float pl = 0.f, xpl = 0.f;
  cs = 1.f;
  // Level l + 1's global inputs are loaded while level l is computed (the
  // loop stays rolled to keep the cloud optics small in the instruction
  // cache).
  float cc_n = F.dcc[c], ql_n = F.dql[c], q_n = absorber(0), t_n = BAND == 0 ? 0.f : F.dt[c], ds_n = ds[0],
        sg_n = sg[0];
#pragma unroll 1
  for (int l = 0; l < NL; ++l) {
    const float cc = cc_n, ql = ql_n, ql_q = q_n, ql_t = t_n, dsl = ds_n, sgl = sg_n;
    if (l + 1 < NL) {
      const size_t at = (l + 1) * SN + c;
      cc_n = F.dcc[at];
      ql_n = F.dql[at];
      q_n = absorber(l + 1);
      t_n = BAND == 0 ? 0.f : F.dt[at];
      ds_n = ds[l + 1];
      sg_n = sg[l + 1];
    }
    float rcl = 0.f, rcls = 0.f, tcl = 1.f, tcls = 1.f;
    if (cc > 0.f) {
      const float lwp = fminf(1000.f, 1000.f * ql * dp / K.GA * dsl);
      const float tau = 2.f * fpow(logf(lwp + 1.5f) * INV_LN10, 3.9f);
      if (BAND == 0) {
        rcls = 1.f - 1.f / (1.f + K.ZB3 * tau);
        const float b1 = K.TSWR1 * sqrtf(mu0);
        const float direct1 = 1.f - 1.f / (1.f + b1 * tau / mu0);
        rcl = cs * direct1 + (1.f - cs) * rcls;
      } else {
        const float zlog = logf(1000.f / tau);
        float b2 = K.ZB4 / logf(3.f + 0.1f * tau);
        float om0 = fminf(0.9999f, 1.f - K.ZB5 * zlog);
        float un = 1.f - om0;
        float uz = un + 2.f * b2 * om0;
        float u = sqrtf(uz / un);
        float ex = expf(fminf(25.f, tau * sqrtf(uz * un) / ZMU00));
        float r = (u + 1.f) * (u + 1.f) * ex - (u - 1.f) * (u - 1.f) / ex;
        tcls = 4.f * u / r;
        rcls = (u * u - 1.f) / r * (ex - 1.f / ex);
        b2 = K.TSWR2 * sqrtf(mu0) / logf(3.f + 0.1f * tau);
        om0 = fminf(0.9999f, 1.f - K.TSWR3 * mu0 * mu0 * zlog);
        un = 1.f - om0;
        uz = un + 2.f * b2 * om0;
        u = sqrtf(uz / un);
        ex = expf(fminf(25.f, tau * sqrtf(uz * un) / mu0));
        r = (u + 1.f) * (u + 1.f) * ex - (u - 1.f) * (u - 1.f) / ex;
        const float directT = 4.f * u / r;
        const float direct2 = (u * u - 1.f) / r * (ex - 1.f / ex);
        tcl = cs * directT + (1.f - cs) * tcls;
        rcl = cs * direct2 + (1.f - cs) * rcls;
      }
    }
    const float amount = amount_of(dsl, ql_q, ql_t, sgl);
    pl = pl + amount;
    xpl = cs * (xpl + zm * amount) + (1.f - cs) * (xpl + diffusivity * amount);
    cs = cs * (1.f - cc);
    lv.at(TL, l) = ta;
    lv.at(RLS, l) = ras;
    const bool surface = l == NL - 1;
    const float tr = (1.f - absorption(xpl)) / tt;
    tt = tt * tr;
    const float tru = ttu / (1.f - absorption(xpt + diffusivity * (pt - pl)));
    ttu = ttu / tru;
    float rb, rbs, tbd, tbu;
    if (BAND == 0) {
      rb = (surface ? rcsSurface : 0.f) + rcl * cc;
      rbs = (surface ? rcsuSurface : 0.f) + rcls * cc;
      tbd = 1.f - (1.f - tr) * (1.f - cc) - rb;
      tbu = 1.f - (1.f - tru) * (1.f - cc) - rbs;
    } else {
      rb = rcl * cc;
      rbs = rcls * cc;
      tbd = 1.f - (1.f - tr) * (1.f - cc) - (1.f - tcl) * cc;
      tbu = 1.f - (1.f - tru) * (1.f - cc) - (1.f - tcls) * cc;
    }
    lv.at(RB, l) = rb;
    lv.at(RBS, l) = rbs;
    lv.at(TBD, l) = tbd;
    lv.at(TBU, l) = tbu;
    const float mm = 1.f / (1.f - ras * rbs);
    ra = ra + ta * rb * tas * mm;
    ta = ta * tbd * mm;
    ras = rbs + tbu * ras * tbd * mm;
    tas = tbu * tas * mm;
  }
  lv.at(TL, NL) = ta;
  lv.at(RLS, NL) = ras;
  // Surface albedo: land and sea ice keep theirs, open water gets a
  // zenith-angle dependent one.
  const bool star = K.NSTARTEMP != 0.f;
  const float dalb = F.dalb[c], salb1 = F.dsalb[c], salb2 = F.dsalb[SN + c];
  const float dls = F.dls[c], dicec = F.dicec[c];
  const float water = (1.f - dls) * (1.f - dicec) * fminf(0.05f / (mu0 + 0.15f), 0.15f);
  const float nalb1 = dls * salb1 + (1.f - dls) * dicec * salb1 + water;
  const float nalb2 = dls * salb2 + (1.f - dls) * dicec * salb2 + water;
  const float albedo = star ? K.ZSOLARS1 * nalb1 + K.ZSOLARS2 * nalb2 : dls * dalb + (1.f - dls) * dicec * dalb + water;
  alb[0] = nalb1;
  alb[1] = nalb2;
  alb[2] = albedo;
  ras = star ? (BAND == 0 ? salb1 : salb2) : dalb;
  ra = star ? (BAND == 0 ? nalb1 : nalb2) : albedo;
  // Upward pass from the surface; level l + 1's flux is complete once its
  // reflectances (ra, ras) are.
#pragma unroll 1
  for (int l = NL - 1; l >= -1; --l) {
    const int k = l + 1;
    const float tl = lv.at(TL, k);
    const float mm = 1.f / (1.f - lv.at(RLS, k) * ras);
    fu[k * stride] = -tl * ra * mm * ftop;
    fd[k * stride] = tl * mm * ftop;
    if (l < 0) break;
    const float rbs = lv.at(RBS, l), tbu = lv.at(TBU, l);
    const float dd = 1.f - ras * rbs;
    ra = lv.at(RB, l) + lv.at(TBD, l) * ra * tbu / dd;
    ras = rbs + tbu * ras * tbu / dd;
  }
}

// swr: the two bands are independent until their fluxes are summed, so the
// block's warps pair up on the same 32 columns, one band each (no branch
// diverges inside a warp), and add their fluxes through shared memory in the
// shader's order (band 1 + band 2).
template <int NL>
__global__ void __launch_bounds__(kBlock) k_swr(Model m) {
  static_assert(NL <= SwrLevels::MAXLEV, "swr level state holds at most MAXLEV levels");
  constexpr int NP = NL + 1;
  constexpr int kCols = kBlock / 2;
  __shared__ float sfu[2][NP][kCols], sfd[2][NP][kCols];
  __shared__ float levels[SwrLevels::kArrays * (SwrLevels::MAXLEV + 1) * kBlock];
  const Dims& d = m.d;
  const int warp = threadIdx.x >> 5;
  const int band = warp & 1;
  const int lc = (warp >> 1) * 32 + (threadIdx.x & 31);
  const int c = blockIdx.x * kCols + lc;
  const bool inside = c < d.S * d.NHOR;
  const int slot = inside ? c / d.NHOR : 0;
  const bool run = inside && m.params[slot].active;
  const PlanetConst& K = m.pc[slot];
  const float* tb = m.tabs + (size_t)slot * m.to.stride;
  const size_t SN = (size_t)d.S * d.NHOR;
  const FieldPtrs& F = m.f;
  bool lit = false;
  float alb[3];
  if (run) {
    const float mu0 = F.gmu0[c];
    const float gdist2 = m.params[slot].rad[3];
    const float ftop1 = K.ZSOLAR1 * K.GSOL0 * gdist2 * mu0;
    const float ftop2 = K.ZSOLAR2 * K.GSOL0 * gdist2 * mu0;
    lit = ftop1 + ftop2 > 1.0e-6f;
    if (lit) {
      const SwrLevels lv{levels};
      if (band == 0)
        swr_band<NL, 0>(m, K, tb, SN, c, mu0, ftop1, lv, &sfu[0][0][lc], &sfd[0][0][lc], kCols, alb);
      else
        swr_band<NL, 1>(m, K, tb, SN, c, mu0, ftop2, lv, &sfu[1][0][lc], &sfd[1][0][lc], kCols, alb);
    }
  }
  __syncthreads();  // both bands' fluxes are in, and both have read dalb, dsalb
  if (!run) return;
  if (lit && band == 0) {
    F.dsalb[c] = alb[0];
    F.dsalb[SN + c] = alb[1];
    F.dalb[c] = alb[2];
  }
  for (int l = band; l < NP; l += 2) {
    float fut = 0.f, fdt = 0.f;
    if (lit) {
      fut = sfu[0][l][lc] + sfu[1][l][lc];
      fdt = sfd[0][l][lc] + sfd[1][l][lc];
    }
    F.dfu[l * SN + c] = fut;
    F.dfd[l * SN + c] = fdt;
    F.dswfl[l * SN + c] = fut + fdt;
  }
}

// lwr (physics/radiation/wgsl/lwr.wgsl) then radstep (radstep.wgsl).
template <int NL>
// Five blocks per SM (at most 102 registers): the kernel is latency-bound;
// five measured faster than six (239 -> 224 us at 128 planets) or seven.
__global__ void __launch_bounds__(kBlock, 5) k_lwr_radstep(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE_STAGED
  const int NP = NL + 1;
  const float ZERO = 1.0e-6f, ZFH2O = 0.1f, ZFO3 = 100.f / 2.14f;
  const float* sg = tb + m.to.sigma;
  const float* sh = tb + m.to.sigmah;
  const float dp = F.dp[c];
  const float ps2 = dp * dp;
  float st4[NL + 1], st4h[NL + 1];
#pragma unroll
  for (int l = 0; l < NP; ++l) {
    const float t = F.dt[l * SN + c];
    const float t2 = t * t;
    st4[l] = K.SBK * (t2 * t2);
  }
  st4h[0] = st4[0] - (st4[0] - st4[1]) * sg[0] / (sg[0] - sg[1]);
#pragma unroll
  for (int l = 1; l < NL; ++l) {
    const float above = sg[l - 1], half = sh[l - 1], level = sg[l];
    st4h[l] = (st4[l] * (above - half) + st4[l - 1] * (half - level)) / (above - level);
  }
  const int n = NL - 1;
  if ((st4[n] - st4h[n]) * (st4[n] - st4[NL]) > 0.f) {
    st4h[NL] = st4[NL];
  } else {
    const float sn = sg[n], sm = sg[n - 1];
    st4h[NL] = st4[n] + (st4[n] - st4[n - 1]) * (1.f - sn) / (sn - sm);
  }
  float bu[NL + 2], bd[NL + 2];
  bd[0] = 0.f;
  const float dls = F.dls[c];
  const float eps = dls + 0.98f * (1.f - dls);
  bu[NP] = eps * st4[NL];
  float q[NL], qo3[NL], qco2[NL], taucc0[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const float sfac = tb[m.to.lwr_zzf1 + l] * ps2;
    q[l] = ZFH2O * sfac * F.dq[l * SN + c];
    qo3[l] = ZFO3 * sfac * F.dqo3[l * SN + c];
    qco2[l] = K.ZFCO2_ZZF2 * sfac * F.dqco2[l * SN + c];
    taucc0[l] = 1.f - F.dcc[l * SN + c] * (1.f - expf(tb[m.to.lwr_zzf3 + l] * F.dql[l * SN + c] * dp));
  }
  // The transmissivity between levels j and k (k >= j) depends on the
  // absorber sums from j down to k. Row j = 0 also sets the layer Planck
  // terms bu, bd; every row j adds its fluxes. The outer loop over j is
  // unrolled (j-indexed values in registers); the inner loop over k stays
  // rolled, reading the absorber amounts, bu and dftd from this thread's
  // column of shared memory ([level][thread], conflict-free, private to the
  // thread), so the code stays small and nothing spills.
  __shared__ float s_q[NL][kBlock], s_o3[NL][kBlock], s_co2[NL][kBlock], s_tc[NL][kBlock];
  __shared__ float s_bu[NL + 2][kBlock], s_dftd[NL + 1][kBlock];
  const int tx = threadIdx.x;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    s_q[l][tx] = q[l];
    s_o3[l][tx] = qo3[l];
    s_co2[l][tx] = qco2[l];
    s_tc[l][tx] = taucc0[l];
  }
#pragma unroll
  for (int l = 0; l < NP; ++l) s_dftd[l][tx] = 0.f;
  // Clear-sky transmissivity for absorber sums (lwr.wgsl's band fits). Each
  // fit is a power law below its threshold and a logarithm above; both
  // sides are written through one base-2 logarithm of the side's argument,
  // x^y = 2^(y log2 x) and log10 x = log10(2) log2 x, so that the columns of
  // a warp, whichever side they take, share one instruction stream (no
  // divergent branches) and two special-function operations per fit. All
  // power-law arguments are positive.
  auto clear_sky = [&](float sumwv, float sumo3, float sumco2) {
    const float LOG10_2 = 0.30102999566398120f, LN_2 = 0.69314718055994531f;
    const bool wv1 = sumwv <= 0.01f, wv2 = sumwv <= 2.f, co2 = sumco2 <= 1.f, o3 = sumo3 <= 0.01f;
    const float lah = fit_log2(sumwv + (wv1 ? 3.59e-5f : 0.01f));
    const float lth = fit_log2(wv2 ? sumwv + 0.0286f : sumwv - 0.6931f);
    const float lco = fit_log2(co2 ? sumco2 + 0.01022f : sumco2);
    const float lo3 = fit_log2(o3 ? sumo3 + 7.0e-5f : sumo3);
    float ah2o = wv1 ? 0.846f * fit_exp2(0.243f * lah) - K.ZH2O0A : 0.24f * (LOG10_2 * lah) + K.ZAH2OC;
    if (K.TH2OC > 0.f) ah2o = fminf(ah2o + (1.f - expf(-K.TH2OC * sumwv)), 1.f);
    const float aco2 = co2 ? 0.0676f * fit_exp2(0.421f * lco) - K.ZCO20 : 0.0546f * (LOG10_2 * lco) + K.ZACO2C;
    const float th2o = wv2 ? 1.f - (0.832f * fit_exp2(0.26f * lth) - K.ZH2O0)
                           : fmaxf(0.f, K.ZTH2OC - 0.1196f * (LN_2 * lth));
    const float ao3 = o3 ? 0.209f * fit_exp2(0.436f * lo3) - K.ZAO30 : 0.0212f * (LOG10_2 * lo3) + K.ZAO3C;
    return fminf(1.f - ZERO, fmaxf(ZERO, 1.f - ah2o - ao3 - aco2 * th2o));
  };
  float dftu[NL + 1], tausf[NL];
  // Row j = 0 (unrolled): transmissivities from the top, then bu, bd.
  {
    float taucs[NL], tau[NL];
    float taucc = 1.f, sumwv = 0.f, sumo3 = 0.f, sumco2 = 0.f;
#pragma unroll
    for (int k = 0; k < NL; ++k) {
      sumwv = sumwv + q[k];
      sumo3 = sumo3 + qo3[k];
      sumco2 = sumco2 + qco2[k];
      const float cs = clear_sky(sumwv, sumo3, sumco2);
      taucs[k] = cs;
      taucc = taucc * taucc0[k];
      tau[k] = cs * taucc;
    }
    float tau0 = 1.f - ZERO;
#pragma unroll
    for (int k = 0; k < NL; ++k) {
      tau0 = taucs[k] / tau0 * taucc0[k] * K.TPOFMT;
      tau0 = fminf(1.f - ZERO, fmaxf(ZERO, tau0));
      if ((st4[k] - st4h[k]) * (st4[k] - st4h[k + 1]) > 0.f) {
        bd[k + 1] = 0.5f * st4[k] + 0.25f * (st4h[k] + st4h[k + 1]);
        bu[k + 1] = bd[k + 1];
      } else {
        bd[k + 1] = (st4h[k + 1] - tau0 * st4h[k]) / (1.f - tau0) - (st4h[k] - st4h[k + 1]) / logf(tau0);
        bu[k + 1] = st4h[k] + st4h[k + 1] - bd[k + 1];
      }
      tau0 = taucs[k];
    }
#pragma unroll
    for (int l = 1; l < NL + 2; ++l) s_bu[l][tx] = bu[l];
    float u = 0.f - bu[1];
    s_dftd[0][tx] = 0.f + bd[0];
    const float bdl = bd[0] - bd[1];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
      u = u - (bu[k + 2] - bu[k + 1]) * tau[k];
      s_dftd[k + 1][tx] = s_dftd[k + 1][tx] + bdl * tau[k];
    }
    dftu[0] = u;
    tausf[0] = tau[NL - 1];
  }
  // Rows j >= 1: one rolled pass over k per row.
#pragma unroll
  for (int j = 1; j < NL; ++j) {
    float taucc = 1.f, sumwv = 0.f, sumo3 = 0.f, sumco2 = 0.f, tau = 0.f;
    float u = 0.f - bu[j + 1];
    s_dftd[j][tx] = s_dftd[j][tx] + bd[j];
    const float bdl = bd[j] - bd[j + 1];
#pragma unroll 1
    for (int k = j; k < NL; ++k) {
      sumwv = sumwv + s_q[k][tx];
      sumo3 = sumo3 + s_o3[k][tx];
      sumco2 = sumco2 + s_co2[k][tx];
      const float cs = clear_sky(sumwv, sumo3, sumco2);
      taucc = taucc * s_tc[k][tx];
      tau = cs * taucc;
      u = u - (s_bu[k + 2][tx] - s_bu[k + 1][tx]) * tau;
      s_dftd[k + 1][tx] = s_dftd[k + 1][tx] + bdl * tau;
    }
    dftu[j] = u;
    tausf[j] = tau;
  }
  float dftd[NL + 1];
#pragma unroll
  for (int l = 0; l < NP; ++l) dftd[l] = s_dftd[l][tx];
  dftu[NL] = 0.f - bu[NP];
  dftd[NL] = dftd[NL] + bd[NL];
  const float reflected = (1.f - eps) * dftd[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) dftu[l] = dftu[l] - tausf[l] * reflected;
  // radstep's inputs are read before the first store (the compiler cannot
  // prove the fields distinct and would otherwise wait for each in turn).
  float sw[NL + 1], tl[NL], ql[NL], dtdt[NL];
#pragma unroll
  for (int l = 0; l < NP; ++l) sw[l] = F.dswfl[l * SN + c];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    tl[l] = F.dt[l * SN + c];
    ql[l] = F.dq[l * SN + c];
    dtdt[l] = F.dtdt[l * SN + c];
  }
  float lw[NL + 1], flux[NL + 1];
#pragma unroll
  for (int l = 0; l < NP; ++l) {
    F.dftu[l * SN + c] = dftu[l];
    F.dftd[l * SN + c] = dftd[l];
    lw[l] = dftu[l] + dftd[l];
    F.dlwfl[l * SN + c] = lw[l];
  }
  // radstep
#pragma unroll
  for (int l = 0; l < NP; ++l) {
    flux[l] = lw[l] + sw[l];
    F.dflux[l * SN + c] = flux[l];
  }
  const float* ds = tb + m.to.dsigma;
  const float* lnsig = tb + m.to.rad_lnsig;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    const float zdh = -tl[l] * K.GASCON / K.GA * lnsig[l];
    const float den = ds[l] * dp * K.ACPD * (1.f + K.ADV * ql[l]);
    F.dtdt[at] = dtdt[l] - K.GA * (flux[l + 1] - flux[l]) / den;
    F.dtdtswr[at] = -K.GA * (sw[l + 1] - sw[l]) / den;
    F.dtdtlwr[at] = -K.GA * (lw[l + 1] - lw[l]) / den;
    F.dconv[at] = (flux[l] - flux[l + 1]) / (zdh + 1.0e-9f);
  }
}

// ---------------------------------------------------------------- precipitation
struct Parcel {
  float t, q, cor;
  bool saturated;
};

// kuo.wgsl's condense: a lifted parcel's two Newton condensation steps.
__device__ __forceinline__ Parcel condense(const PlanetConst& K, float t0, float q0, float p) {
  float s = sat_capped(K, t0, p);
  float cor = 1.f / (1.f - K.MOIST * s);
  s = s * cor;
  if (!(s < q0)) return {t0, q0, cor, false};
  float t = t0, q = q0;
  const float lcp = (t0 < K.TMELT ? K.ALS : K.ALV) / (K.ACPD * (1.f + K.ADV * q0));
  for (int i = 0; i < 2; ++i) {
    if (i == 1) {
      s = sat_capped(K, t, p);
      cor = 1.f / (1.f - K.MOIST * s);
      s = s * cor;
    }
    const float dqsdt = K.RA2 * (K.TMELT - K.RA4) * s * cor / ((t - K.RA4) * (t - K.RA4));
    const float rain = (q - s) / (1.f + lcp * dqsdt);
    t = t + lcp * rain;
    q = q - rain;
  }
  return {t, q, cor, true};
}

// mkdqtgp scaling, kuo and mkshallow (physics/precipitation/wgsl/kuo.wgsl).
// Four resident blocks per SM: with the restrict parameters the compiler
// keeps more values in registers, and four blocks measured faster than six
// or three.
template <int NL>
__device__ __forceinline__ void b_kuo(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const int NM = NL - 1;
  const float* ds = tb + m.to.dsigma;
  const float* sg = tb + m.to.sigma;
  const float D2 = P.deltsec2;
  const float dp = F.dp[c];
  float zdqt[NL], zqe[NL], zte[NL], zdqtot[NL], zalcpe[NL], zacpe[NL], zdqdt[NL], zdtdt[NL];
  // Every field this column reads is loaded before its first store (the
  // compiler cannot prove the fields distinct, and would otherwise wait for
  // each later load in turn); dtdt and dqdt stay in registers.
  float dqt_in[NL], dq_in[NL], dqdt_in[NL], dt_in[NL], dtdt_in[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    dqt_in[l] = F.dqt[at];
    dq_in[l] = F.dq[at];
    dqdt_in[l] = F.dqdt[at];
    dt_in[l] = F.dt[at];
    dtdt_in[l] = F.dtdt[at];
  }
  const float dt_surface = F.dt[NL * SN + c], dq_surface = F.dq[NL * SN + c];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    zdqt[l] = dqt_in[l] * K.PSURF * K.WW / dp;
    F.dqt[at] = zdqt[l];
    const float dq = dq_in[l], dqdt = dqdt_in[l];
    zdqtot[l] = (zdqt[l] + dqdt) * D2;
    zqe[l] = dq + dqdt * D2;
    zte[l] = dt_in[l] + dtdt_in[l] * D2;
    zacpe[l] = K.ACPD * (1.f + K.ADV * dq);
    zalcpe[l] = K.ALV / zacpe[l];
    zdqdt[l] = 0.f;
    zdtdt[l] = 0.f;
  }
  int ilift = -1, itop = -1;
  float zi = 0.f, zpt = 0.f, zpq = 0.f, zbeta = 0.f, zpbeta = 0.f, ztp = 0.f, zqp = 0.f;
  {
    const int n = NL - 1;
    const float dsn = ds[n];
    const float ztsurf = dt_surface * tb[m.to.vdiff_skap + n];
    if (zdqtot[n] > 0.f && ztsurf > zte[n]) {
      const float p = dp * sg[n];
      const float zqsnl = sat_divided(K, zte[n], p);
      const float zqnew = dq_surface * fminf(1.f, zqe[n] / zqsnl);
      const Parcel parcel = condense(K, ztsurf, zqnew, p);
      if (parcel.saturated) {
        ilift = NL + 1;
        itop = NL;
        ztp = parcel.t;
        zqp = parcel.q;
        const float zqsa = sat_divided(K, zte[n], p);
        zdqdt[n] = fmaxf(zqsa - zqe[n], 0.f);
        zdtdt[n] = ztp - zte[n];
        zpt = zdtdt[n] * dsn * zacpe[n];
        zpq = zdqdt[n] * dsn * K.ALV;
        zbeta = fminf(1.f, zqe[n] / zqsa) * dsn;
        zpbeta = dsn;
        zi = zdqtot[n] * dsn * K.ALV;
      }
    }
  }
  // Both level loops are unrolled: a rolled loop would index the per-level
  // arrays at run time and keep them in local memory.
#pragma unroll
  for (int l = NM - 1; l >= 0; --l) {
    const int lp = l + 1;
    if (ilift == -1 && zdqtot[lp] > 0.f) {
      const float p = dp * sg[l];
      const Parcel parcel = condense(K, zte[lp] * tb[m.to.kuo_zfac + l], zqe[lp], p);
      if (parcel.saturated && parcel.t > zte[l]) {
        const float dsl = ds[l], dsp = ds[lp];
        ilift = l + 2;
        itop = l + 1;
        ztp = parcel.t;
        zqp = parcel.q;
        const float zqsa = sat_divided(K, zte[l], p);
        zdqdt[l] = fmaxf(zqsa - zqe[l], 0.f);
        zdtdt[l] = ztp - zte[l];
        zpt = zdtdt[l] * dsl * zacpe[l];
        zpq = zdqdt[l] * dsl * K.ALV;
        zbeta = fminf(1.f, zqe[l] / zqsa) * dsl;
        zpbeta = dsl;
        const float pp = dp * sg[lp];
        float zqsnl = sat_divided(K, zte[lp], pp);
        if (zqe[lp] > zqsnl) {
          float t = zte[lp], q = zqe[lp];
          const float lcp = (t < K.TMELT ? K.ALS : K.ALV) / (K.ACPD * (1.f + K.ADV * q));
          float cor = parcel.cor;
          for (int i = 0; i < 2; ++i) {
            if (i == 1) {
              zqsnl = sat_capped(K, t, pp);
              cor = 1.f / (1.f - K.MOIST * zqsnl);
              zqsnl = zqsnl * cor;
            }
            const float dqsdt = K.RA2 * (K.TMELT - K.RA4) * zqsnl * cor / ((t - K.RA4) * (t - K.RA4));
            const float rain = (q - zqsnl) / (1.f + lcp * dqsdt);
            t = t + lcp * rain;
            q = q - rain;
          }
          zdqdt[lp] = fmaxf(q - zqe[lp], 0.f);
          zdtdt[lp] = t - zte[lp];
          zpt = zdtdt[lp] * dsp * zacpe[lp] + zpt;
          zpq = zdqdt[lp] * dsp * K.ALV + zpq;
          zbeta = fminf(1.f, zqe[lp] / zqsnl) * dsp + zbeta;
          zpbeta = dsp + zpbeta;
        }
        zi = zdqtot[l] * dsl * K.ALV + zdqtot[lp] * dsp * K.ALV;
      }
    }
  }
#pragma unroll
  for (int l = NM - 1; l >= 0; --l) {
    if (itop == l + 2) {
      const float p = dp * sg[l];
      const Parcel parcel = condense(K, ztp * tb[m.to.kuo_zfac + l], zqp, p);
      if (parcel.saturated && parcel.t > zte[l]) {
        const float dsl = ds[l];
        itop = l + 1;
        ztp = parcel.t;
        zqp = parcel.q;
        const float zqsa = sat_divided(K, zte[l], p);
        zdqdt[l] = fmaxf(zqsa - zqe[l], 0.f);
        zdtdt[l] = ztp - zte[l];
        zpt = zdtdt[l] * dsl * zacpe[l] + zpt;
        zpq = zdqdt[l] * dsl * K.ALV + zpq;
        zbeta = fminf(1.f, zqe[l] / zqsa) * dsl + zbeta;
        zpbeta = zpbeta + dsl;
        zi = zdqtot[l] * dsl * K.ALV + zi;
      }
    }
  }
  zi = fmaxf(0.f, zi);
  const float zrhm = zpbeta > 0.f ? zbeta / zpbeta : 0.f;
  float beta = 1.f;
  if (zrhm >= K.RHBETA) beta = powi((1.f - zrhm) / (1.f - K.RHBETA), (int)K.NBETA);
  const float zat = zpt > 0.f ? zi * (1.f - beta) / zpt : 0.f;
  const float zaq = zpq > 0.f ? zi * beta / zpq : 0.f;
  const bool shallow = itop > 0 && (dp * sg[itop - 1] > K.PDEEP || zi <= 0.f);
  float icctot = 0.f;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const int level = l + 1;
    const size_t at = l * SN + c;
    float dprcl = 0.f, icclev = 0.f;
    if (ilift >= level && itop <= level && zi > 0.f && !shallow) {
      F.dqdt[at] = zaq * zdqdt[l] / D2 - zdqt[l];
      F.dtdt[at] = zat * zdtdt[l] / D2 + dtdt_in[l];
      dprcl = zat * zdtdt[l] * ds[l] / zalcpe[l] / D2;
    }
    if (dprcl > 0.f) {
      icclev = 1.f;
      icctot = icctot + 1.f;
    }
    if (sg[l] < 0.4f && icclev == 1.f && itop == level) icclev = 2.f;
    F.dprcl[at] = dprcl;
    F.dprscl[at] = 0.f;
    F.icclev[at] = icclev;
  }
  F.icctot[c] = icctot;
  if (!shallow) return;
  const float zkonst1 = K.GA * D2 / K.GASCON;
  const float zkonst2 = K.RKSHALLOW * zkonst1 * K.GA / K.GASCON;
  int kktop = 1;
  for (int level = 2; level <= NM; ++level)
    if (dp * sg[level - 1] < K.PDEEPTH) kktop = level;
  const int ktop = max(itop, kktop);
  float zkdiff[NL], skap[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    zkdiff[l] = 0.f;
    skap[l] = tb[m.to.vdiff_skap + l];
  }
#pragma unroll
  for (int l = 0; l < NM; ++l) {
    const int lp = l + 1, level = l + 1;
    const float sigmah = tb[m.to.sigmah + l];
    const float zfac = zkonst2 * sigmah * sigmah * tb[m.to.vdiff_rdsig + l];
    const float dsl = ds[l], dsp = ds[lp];
    const float zrthl = (dsp + dsl) / (zte[l] * dsp + zte[lp] * dsl);
    if (level >= ktop && level < ilift) zkdiff[l] = zfac * zrthl * zrthl;
    if (level + 1 == ktop) {
      float zzqs = sat_capped(K, zte[l], dp * sg[l]);
      zzqs = zzqs * (1.f / (1.f - K.MOIST * zzqs));
      float zzqsp = sat_capped(K, zte[lp], dp * sg[lp]);
      zzqsp = zzqsp * (1.f / (1.f - K.MOIST * zzqsp));
      const float zrh = zqe[l] / zzqs, zrhp = zqe[lp] / zzqsp;
      const float zzf = fabsf((zrh - 0.8f) / 0.2f * (zrhp - zrh));
      zkdiff[l] = zfac * zrthl * zrthl * zzf;
    }
  }
  float zqn[NL], ztn[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    zqn[l] = zqe[l];
    ztn[l] = zte[l];
  }
  diffuse<NL>(ds, zqn, zkdiff);
#pragma unroll
  for (int l = 0; l < NM; ++l) zkdiff[l] = zkdiff[l] * tb[m.to.vdiff_skaph + l];
  diffuse_potential<NL>(ds, ztn, zkdiff, skap);
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    // a shallow column's deep-convection writes above did not run
    const size_t at = l * SN + c;
    F.dtdt[at] = dtdt_in[l] + (ztn[l] - zte[l]) / D2;
    F.dqdt[at] = dqdt_in[l] + (zqn[l] - zqe[l]) / D2;
  }
}
template <int NL>
__global__ void __launch_bounds__(kBlock, 4) k_kuo(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_kuo<NL>(m, pcr, tabr);
}


// mkdca (physics/precipitation/wgsl/mkdca.wgsl): dry convective adjustment.
template <int NL>
__device__ __forceinline__ void b_mkdca(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const int NM = NL - 1;
  const float D2 = P.deltsec2;
  float zt[NL], zth[NL], zq[NL], zqn[NL], skap[NL], ds[NL];
  bool mixed[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    skap[l] = tb[m.to.vdiff_skap + l];
    ds[l] = tb[m.to.dsigma + l];
    zt[l] = F.dt[at] + F.dtdt[at] * D2;
    zth[l] = zt[l] / skap[l];
    zq[l] = F.dq[at] + F.dqdt[at] * D2;
    zqn[l] = zq[l];
    mixed[l] = false;
  }
  float limited = 0.f;
  int passes = 0;
  for (;;) {
    bool unstable = false;
    int ibase = 0, itop = NL;
    float ztht = 0.f, zqt = 0.f, zsum1 = 0.f, zsum2 = 0.f, zsumq1 = 0.f, zsumq2 = 0.f;
    for (int l = 0; l < NM; ++l) {
      const int lp = l + 1;
      if (zth[l] < zth[lp]) {
        ibase = l + 2;
        itop = l;
        zsum1 = skap[lp] * ds[lp] + skap[l] * ds[l];
        zsum2 = skap[lp] * ds[lp] * zth[lp] + skap[l] * ds[l] * zth[l];
        zsumq1 = ds[lp] + ds[l];
        zsumq2 = ds[lp] * zqn[lp] + ds[l] * zqn[l];
        ztht = zsum2 / zsum1;
        zqt = zsumq2 / zsumq1;
        unstable = true;
      }
    }
    if (!unstable) break;
    for (int level = NM - 1; level >= 1; --level) {
      const int l = level - 1;
      if (itop == level && zth[l] < ztht) {
        itop = level - 1;
        zsum1 = zsum1 + skap[l] * ds[l];
        zsum2 = zsum2 + skap[l] * ds[l] * zth[l];
        zsumq1 = zsumq1 + ds[l];
        zsumq2 = zsumq2 + ds[l] * zqn[l];
        ztht = zsum2 / zsum1;
        zqt = zsumq2 / zsumq1;
      }
    }
    for (int l = 0; l < NL; ++l) {
      const int level = l + 1;
      if (level > itop && level <= ibase) {
        zth[l] = ztht;
        zqn[l] = zqt;
        mixed[l] = true;
      }
    }
    passes = passes + 1;
    if (passes > 2 * NL) {  // the reference's pass limit bounds this loop
      limited = 1.f;
      break;
    }
  }
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    F.dca_dtdt[at] = mixed[l] ? (zth[l] * skap[l] - zt[l]) / D2 : 0.f;
    F.dca_dqdt[at] = (zqn[l] - zq[l]) / D2;
  }
  F.dca_limited[c] = limited;
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_mkdca(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_mkdca<NL>(m, pcr, tabr);
}


// mkdca-limit (physics/precipitation/wgsl/mkdca-limit.wgsl): per slot, skip
// every adjustment when any column needed more than 2 NL passes.
__global__ void __launch_bounds__(kSumThreads) k_mkdca_limit(Model m) {
  const Dims& d = m.d;
  const int slot = blockIdx.x;
  if (!m.params[slot].active) return;
  __shared__ float part[kSumThreads];
  float flag = 0.f;
  for (int h = threadIdx.x; h < d.NHOR; h += kSumThreads) flag = fmaxf(flag, m.f.dca_limited[slot * d.NHOR + h]);
  part[threadIdx.x] = flag;
  __syncthreads();
  for (int stride = kSumThreads / 2; stride > 0; stride /= 2) {
    if (threadIdx.x < stride) part[threadIdx.x] = fmaxf(part[threadIdx.x], part[threadIdx.x + stride]);
    __syncthreads();
  }
  if (threadIdx.x == 0) m.f.dca_skip[slot] = part[0];
}

// column.wgsl: mkdca's adjustment (unless skipped), mklsp, mkrain, mkclouds.
// Its parameters carry no __restrict__: with it the compiler keeps more
// values in registers (165), and the lower occupancy measured slower. The
// planet's constants, read again after the stores of each level loop, sit
// in shared memory (259 -> 252 us per launch at 128 T42 L10 planets).
template <int NL>
__device__ __forceinline__ void b_rain_column(const Model& m, const PlanetConst* pcr, const float* tabr) {
  COLUMN_PROLOGUE_STAGED
  const float* ds = tb + m.to.dsigma;
  const float* sg = tb + m.to.sigma;
  const float D2 = P.deltsec2;
  const bool skip = F.dca_skip[slot] != 0.f;
  const float dp = F.dp[c];
  // mkrain's and mkclouds' inputs are read after mklsp's stores; registers
  // cannot hold them from here, so they are fetched into L2 now.
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    prefetch_l2(F.dprscl + at);
    prefetch_l2(F.dprcl + at);
    prefetch_l2(F.icclev + at);
    if (K.CLWFAC > 0.f) prefetch_l2(F.dw + at);
  }
  prefetch_l2(F.icctot + c);
  prefetch_l2(F.dt + NL * SN + c);
  float dq_[NL], dt_[NL], dtdt_[NL], dqdt_[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    dq_[l] = F.dq[at];
    dt_[l] = F.dt[at];
    dtdt_[l] = F.dtdt[at];
    dqdt_[l] = F.dqdt[at];
    if (!skip) {
      dtdt_[l] = dtdt_[l] + F.dca_dtdt[at];
      dqdt_[l] = dqdt_[l] + F.dca_dqdt[at];
    }
  }
  // mklsp
  float dprll[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    dprll[l] = 0.f;
    const float dq = dq_[l];
    const float zq = dq + dqdt_[l] * D2;
    const float zt = dt_[l] + dtdt_[l] * D2;
    // IEEE divisions here (the file otherwise divides to 2 ulp): the
    // large-scale precipitation is the difference of two iterated states.
    const float zlcpe = __fdiv_rn(K.ALV, K.ACPD * (1.f + K.ADV * dq));
    const float p = dp * sg[l];
    float zqsat = sat_capped_rn(K, zt, p);
    float zcor = __fdiv_rn(1.f, 1.f - K.MOIST * zqsat);
    zqsat = zqsat * zcor;
    if (zqsat < 0.f) zqsat = 0.f;
    if (zq > zqsat) {
      float zdqdt = __fdiv_rn(zqsat - zq, 1.f + __fdiv_rn(zlcpe * K.RA2 * (K.TMELT - K.RA4) * zqsat * zcor,
                                                          (zt - K.RA4) * (zt - K.RA4)));
      float ztn = zt - zdqdt * zlcpe;
      float zqn = zq + zdqdt;
      zqsat = sat_capped_rn(K, ztn, p);
      zcor = __fdiv_rn(1.f, 1.f - K.MOIST * zqsat);
      zqsat = zqsat * zcor;
      zdqdt = __fdiv_rn(zqsat - zqn, 1.f + __fdiv_rn(zlcpe * K.RA2 * (K.TMELT - K.RA4) * zqsat * zcor,
                                                     (ztn - K.RA4) * (ztn - K.RA4)));
      ztn = ztn - zdqdt * zlcpe;
      zqn = zqn + zdqdt;
      const float dqdt = __fdiv_rn(zqn - zq, D2), dtdt = __fdiv_rn(ztn - zt, D2);
      dqdt_[l] = dqdt_[l] + dqdt;
      dtdt_[l] = dtdt_[l] + dtdt;
      dprll[l] = -fminf(dqdt, 0.f) * ds[l];
    }
    F.dprsll[l * SN + c] = 0.f;
    F.dprll[l * SN + c] = dprll[l];
  }
  // mkrain
  float zprc = 0.f, zprl = 0.f, zprsc = 0.f, zprsl = 0.f;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    const float dsl = ds[l], dq = dq_[l];
    float zdtdt = 0.f, zdqdtl = 0.f, zdqdts = 0.f;
    const float dprscl = F.dprscl[at];
    zprc = zprc + F.dprcl[at] - dprscl;
    zprl = zprl + dprll[l] - 0.f;
    zprsc = zprsc + dprscl;
    zprsl = zprsl + 0.f;
    const int surface = l == NL - 1 ? 2 : 1;
    for (int below = 0; below < surface; ++below) {
      const float temperature = F.dt[(l + below) * SN + c];
      const float zlcp = (K.ALS - K.ALV) / (K.ACPD * (1.f + K.ADV * dq));
      if (zprsc + zprsl > 0.f && temperature > K.TMELT) {
        zdtdt = -(zprsc + zprsl) / dsl * zlcp + zdtdt;
        zprc = zprsc + zprc;
        zprl = zprsl + zprl;
        zprsc = 0.f;
        zprsl = 0.f;
      } else if (zprc + zprl > 0.f && temperature <= K.TMELT) {
        zdtdt = (zprc + zprl) / dsl * zlcp + zdtdt;
        zprsc = zprc + zprsc;
        zprsl = zprl + zprsl;
        zprc = 0.f;
        zprl = 0.f;
      }
    }
    const float zq = dq + dqdt_[l] * D2;
    const float zt = dt_[l] + dtdt_[l] * D2;
    float zqsat = sat_capped(K, zt, dp * sg[l]);
    const float zcor = 1.f / (1.f - K.MOIST * zqsat);
    zqsat = zqsat * zcor;
    if (zqsat < 0.f) zqsat = 0.f;
    if (zq < zqsat) {
      const float deficit = zqsat - zq;
      const float water = K.ALV / (K.ACPD * (1.f + K.ADV * dq));
      const float ice = K.ALS / (K.ACPD * (1.f + K.ADV * dq));
      const float curve = K.RA2 * (K.TMELT - K.RA4) * zqsat * zcor / ((zt - K.RA4) * (zt - K.RA4));
      auto evap = [&](float& flux, float zlcpe) {
        const float zd = fminf(K.GAMMA * deficit * dsl / D2 / (1.f + zlcpe * curve), flux);
        flux = flux - zd;
        return zd / dsl;
      };
      if (zprl > 0.f) {
        const float e = evap(zprl, water);
        zdtdt = zdtdt - e * water;
        zdqdtl = zdqdtl + e;
      }
      if (zprc > 0.f) {
        const float e = evap(zprc, water);
        zdtdt = zdtdt - e * water;
        zdqdtl = zdqdtl + e;
      }
      if (zprsl > 0.f) {
        const float e = evap(zprsl, ice);
        zdtdt = zdtdt - e * ice;
        zdqdts = zdqdts + e;
      }
      if (zprsc > 0.f) {
        const float e = evap(zprsc, ice);
        zdtdt = zdtdt - e * ice;
        zdqdts = zdqdts + e;
      }
    }
    dqdt_[l] = dqdt_[l] + zdqdtl + zdqdts;
    dtdt_[l] = dtdt_[l] + zdtdt;
  }
  const float dprc = (zprc + zprsc) * dp / K.GA / 1000.f;
  F.dprc[c] = dprc;
  F.dprl[c] = (zprl + zprsl) * dp / K.GA / 1000.f;
  F.dprs[c] = (zprsc + zprsl) * dp / K.GA / 1000.f;
  // mkclouds
  const float ZCLMAX = 1.f, ZCCA = 0.245f, ZCCB = 0.125f, ZCCMAX = 0.8f, ZCCMIN = 0.05f;
  float zcctot = ZCCMIN, zccconv = ZCCMIN;
  if (dprc > 0.f) {
    zcctot = ZCCA + ZCCB * logf(dprc * K.ZRFAC);
    zcctot = fminf(ZCCMAX, fmaxf(ZCCMIN, zcctot));
    const float levels = F.icctot[c];
    zccconv = levels == 0.f ? 1.f : 1.f - fpow(1.f - zcctot, 1.f / levels);
  }
  float cover[NL];
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    const float zt = dt_[l] + dtdt_[l] * D2;
    const float zq = dq_[l] + dqdt_[l] * D2;
    const float zqsat = sat_divided(K, zt, dp * sg[l]);
    float zrh = zq / zqsat;
    const float icclev = F.icclev[at];
    float dcc = icclev > 0.f ? zccconv : 0.f;
    if (icclev == 2.f && zcctot >= 0.3f) dcc = fminf(dcc + 2.f * (zcctot - 0.3f), ZCLMAX);
    zrh = zrh * (1.f - dcc);
    const float zrcrit = tb[m.to.rcrit + l];
    float zwfac = 1.f;
    if (sg[l] > 0.8f && K.CLWFAC > 0.f) {
      const float dw = F.dw[at];
      zwfac = K.CLWFAC * fmaxf(0.f, K.CLWCRIT1 - dw);
      if (K.CLWCRIT2 > dw) zwfac = 1.f;
    }
    const float excess = fmaxf(0.f, (zrh - zrcrit) / (1.f - zrcrit));
    cover[l] = fminf(dcc + zwfac * (excess * excess), ZCLMAX);
  }
  const float* lnsig = tb + m.to.rad_lnsig;
  float zzf[NL];
  float dqvi = 0.f, zzh = 0.f;
#pragma unroll
  for (int l = NL - 1; l >= 1; --l) {
    dqvi = dq_[l] * ds[l] + dqvi;
    const float zdh = -dt_[l] * K.GASCON / K.GA * lnsig[l];
    zzf[l] = zzh + zdh * 0.5f;
    zzh = zzh + zdh;
  }
  dqvi = dq_[0] * ds[0] + dqvi;
  zzf[0] = zzh - dt_[0] * K.GASCON / K.GA * lnsig[0];
  dqvi = dqvi * dp / K.GA;
  F.dqvi[c] = dqvi;
  zzh = 700.f * logf(1.f + dqvi);
  float clear = 1.f;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const size_t at = l * SN + c;
    float dql = 0.f;
    if (zzh > 0.f && cover[l] > 0.f) {
      dql = 0.00021f * expf(-zzf[l] / zzh) * K.GASCON * dt_[l] / (sg[l] * dp);
      dql = fmaxf(dql, 1.0e-9f);
    }
    F.dql[at] = dql;
    F.dcc[at] = cover[l];
    F.dtdt[at] = dtdt_[l];
    F.dqdt[at] = dqdt_[l];
    clear = clear * (1.f - cover[l]);
  }
  F.dql[NL * SN + c] = 0.f;
  F.dcc[NL * SN + c] = 1.f - clear;
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_rain_column(Model m, const PlanetConst* pcr, const float* tabr) {
  b_rain_column<NL>(m, pcr, tabr);
}


// ---------------------------------------------------------------- surface
struct SnowLayer {
  float ctop, soilz1, diff1, cap1;
};

__device__ __forceinline__ SnowLayer snow_layer(const PlanetConst& K, float snowz, float cap0, float diff0,
                                                float soilz0) {
  const float zsntop = fminf(snowz * 1000.f / K.RHOSNOW, K.DZTOP);
  const float ctop = cap0 * K.SNOWCAP * K.DZTOP / (cap0 * zsntop + K.SNOWCAP * (K.DZTOP - zsntop));
  const float zsnowz = fminf(snowz * 1000.f / K.RHOSNOW, 1.f) - zsntop;
  const float soilz1 = soilz0 + zsnowz;
  const float diff1 = diff0 * K.SNOWDIFF * soilz1 / (K.SNOWDIFF * soilz0 + diff0 * zsnowz);
  const float cap1 = cap0 * K.SNOWCAP * soilz1 / (cap0 * zsnowz + K.SNOWCAP * soilz0);
  return {ctop, soilz1, diff1, cap1};
}

__device__ __forceinline__ float surface_temperature(const PlanetConst& K, float deltsec, const SnowLayer& ly,
                                                     float dtsm, float flux, float soil1) {
  const float conduction = 2.f * ly.diff1;
  return (ly.ctop * K.DZTOP * dtsm / deltsec + flux + conduction * soil1 / ly.soilz1) /
         (ly.ctop * K.DZTOP / deltsec + conduction / ly.soilz1);
}

// landmod's soilstep (physics/land/wgsl/soil.wgsl): tands, mktsoil, wandr.
template <int NL>
__device__ __forceinline__ void b_soil(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const float DS = P.deltsec;
  const float dls = F.dls[c];
  const bool land = dls > 0.f;
  const float snowStart = F.dsnowz[c];
  // Every input is read before the first store (the compiler cannot prove
  // the fields distinct, so a store would order each later load after it):
  // the snow temperature is stored at the end, and the bucket's water and
  // capacity are read here.
  const float dwatc_in = land ? F.dwatc[c] : 0.f, dwmax = land ? F.dwmax[c] : 0.f;
  float dwater = 0.f, dsmelt = 0.f;
  bool put_snowt = snowStart == 0.f;
  float snowt = K.TMELT;
  if (land) {
    const float glac = F.dglac[c];
    float soilz[NLSOIL], cap[NLSOIL], diff[NLSOIL];
#pragma unroll
    for (int l = 0; l < NLSOIL; ++l) {
      cap[l] = K.SICECAP * glac + K.SOILCAP * (1.f - glac);
      diff[l] = K.SICEDIFF * glac + K.SOILDIFF * (1.f - glac);
      soilz[l] = tb[m.to.dsoilz + l];
    }
    const float zhfla = F.dshfl[c] + F.dlhfl[c] + F.dflux[NL * SN + c];
    const float devap = F.devap[c];
    float zdsnowz = 0.f;
    if (F.dprs[c] > 0.f) zdsnowz = F.dprs[c];
    if (snowStart > 0.f) zdsnowz = zdsnowz + devap;
    float zsnowz = fmaxf(0.f, snowStart + zdsnowz * DS);
    zdsnowz = (zsnowz - snowStart) / DS;
    dwater = devap + F.dprl[c] + F.dprc[c] - zdsnowz;
    float dsnowz = zsnowz;
    const float dtsm = F.land_dtsm[c];
    const float soil1 = F.dsoilt[c];
    SnowLayer layer = snow_layer(K, dsnowz, cap[0], diff[0], soilz[0]);
    float dts = surface_temperature(K, DS, layer, dtsm, zhfla, soil1);
    float zhfls = 2.f * layer.diff1 / layer.soilz1 * (dts - soil1);
    float zhflm = 0.f;
    if (dsnowz > 0.f && dts > K.TMELT) {
      dts = K.TMELT;
      zhflm = fmaxf(0.f, zhfla - layer.ctop * K.DZTOP * (dts - dtsm) / DS + 2.f * layer.diff1 * (soil1 - dts) / layer.soilz1);
      zsnowz = fmaxf(0.f, dsnowz - zhflm * DS / ((K.ALS - K.ALV) * 1000.f));
      zdsnowz = (zsnowz - dsnowz) / DS;
      zhflm = -zdsnowz * 1000.f * (K.ALS - K.ALV);
      dsnowz = zsnowz;
      dsmelt = -zdsnowz;
      zhfls = 2.f * layer.diff1 / layer.soilz1 * (dts - soil1);
      dwater = dwater - zdsnowz;
      layer = snow_layer(K, dsnowz, cap[0], diff[0], soilz[0]);
    }
    if (dsnowz == 0.f && zhflm > 0.f) {
      dts = surface_temperature(K, DS, layer, dtsm, zhfla - zhflm, soil1);
      zhfls = 2.f * layer.diff1 / layer.soilz1 * (dts - soil1);
    }
    soilz[0] = layer.soilz1;
    cap[0] = layer.cap1;
    diff[0] = layer.diff1;
    // mktsoil
    float zdiff[NLSOIL], zcap[NLSOIL], zebs[NLSOIL], ztn[NLSOIL];
    const int n = NLSOIL - 1;
    zdiff[n - 1] = 2.f * diff[n] * diff[n - 1] / (diff[n] * soilz[n - 1] + diff[n - 1] * soilz[n]);
    zcap[n] = cap[n] * soilz[n] / DS;
    zebs[n] = 1.f / (zcap[n] + zdiff[n - 1]);
    ztn[n] = zcap[n] * F.dsoilt[n * SN + c] * zebs[n];
#pragma unroll
    for (int l = n - 1; l >= 1; --l) {
      zdiff[l - 1] = 2.f * diff[l] * diff[l - 1] / (diff[l] * soilz[l - 1] + diff[l - 1] * soilz[l]);
      zcap[l] = cap[l] * soilz[l] / DS;
      zebs[l] = 1.f / (zcap[l] + zdiff[l - 1] + zdiff[l] * (1.f - zdiff[l] * zebs[l + 1]));
      ztn[l] = zebs[l] * (zcap[l] * F.dsoilt[l * SN + c] + zdiff[l] * ztn[l + 1]);
    }
    zcap[0] = cap[0] * soilz[0] / DS;
    zebs[0] = 1.f / (zcap[0] + zdiff[0] * (1.f - zdiff[0] * zebs[1]));
    ztn[0] = zebs[0] * (zcap[0] * F.dsoilt[c] + zdiff[0] * ztn[1] + zhfls);
#pragma unroll
    for (int l = 1; l < NLSOIL; ++l) ztn[l] = ztn[l] + zebs[l] * zdiff[l - 1] * ztn[l - 1];
    const bool glacier = F.dglac[c] > 0.5f;
#pragma unroll
    for (int l = 0; l < NLSOIL; ++l) F.dsoilt[l * SN + c] = glacier ? fminf(ztn[l], K.TMELT) : ztn[l];
    if (dsnowz > 0.f) {
      snowt = dts;
      put_snowt = true;
    }
    if (K.DSMAX > 0.f && dsnowz > K.DSMAX) {
      zdsnowz = (K.DSMAX - dsnowz) / DS;
      dsnowz = K.DSMAX;
      dwater = dwater - zdsnowz;
      dts = dts + zdsnowz * 1000.f * (K.ALS - K.ALV) * DS / layer.ctop / K.DZTOP;
      dsmelt = dsmelt - zdsnowz;
    }
    F.dsnowz[c] = dsnowz;
    F.land_dts[c] = dts;
    F.dsndch[c] = dsnowz - snowStart;
  } else {
    F.dsndch[c] = snowStart;
  }
  F.dwater[c] = dwater;
  F.dsmelt[c] = dsmelt;
  float drunoff = 0.f;
  if (land) {
    const float dwatc = dwatc_in + DS * dwater;
    drunoff = fmaxf(0.f, dwatc - dwmax) / DS;
    F.dwatc[c] = fmaxf(fminf(dwmax, dwatc), 0.f);
  }
  F.drunoff[c] = drunoff;
  if (put_snowt) F.dsnowt[c] = snowt;
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_soil(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_soil<NL>(m, pcr, tabr);
}


// mkradv (physics/land/wgsl/mkradv.wgsl): river routing stencil within one
// slot. Each thread reads only its own drunoff and its neighbours' driver,
// which nothing here writes, so the update is in place.
__device__ __forceinline__ float river(const FieldPtrs& F, int c) { return F.driver[c] * F.darea[c] * F.dls[c]; }

__global__ void __launch_bounds__(kBlock) k_mkradv(Model m) {
  const Dims& d = m.d;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.S * d.NHOR) return;
  const int slot = c / d.NHOR, h = c % d.NHOR;
  if (!m.params[slot].active) return;
  const FieldPtrs& F = m.f;
  const int base = slot * d.NHOR;
  const int lat = h / d.NLON, lon = h % d.NLON;
  const int row = base + lat * d.NLON;
  auto eastward = [&](int lo, float& out, float& into) {
    const int at = row + lo, nx = row + (lo + 1) % d.NLON;
    const float u = F.duroff[at];
    const float water = u > 0.f ? river(F, at) : river(F, nx);
    out = u * water / F.darea[at];
    into = u * water / F.darea[nx];
  };
  float runoff = F.drunoff[c], o, in;
  if (lon == 0) {
    eastward(0, o, in);
    runoff = runoff - o;
    eastward(d.NLON - 1, o, in);
    runoff = runoff + in;
  } else {
    eastward(lon - 1, o, in);
    runoff = runoff + in;
    eastward(lon, o, in);
    runoff = runoff - o;
  }
  const float area = F.darea[c], v = F.dvroff[c];
  const float below = lat + 1 < d.NLAT ? river(F, c + d.NLON) : 0.f;
  if (v < 0.f)
    runoff = runoff + v * river(F, c) / area;
  else
    runoff = runoff + v * below / area;
  float fromAbove = 0.f;
  if (lat > 0) {
    const int above = c - d.NLON;
    const float va = F.dvroff[above];
    fromAbove = va < 0.f ? -va * river(F, above) : -va * river(F, c);
  }
  F.drunoff[c] = runoff + fromAbove / area;
}

__device__ __forceinline__ float clim14(const float* f, const float* w3, int c, size_t SN) {
  const float w = w3[2];
  return (1.f - w) * f[(size_t)w3[0] * SN + c] + w * f[(size_t)w3[1] * SN + c];
}

// Land surface after mkradv (physics/land/wgsl/surface.wgsl) with vegstep
// (vegetation/wgsl/vegstep.wgsl) and glacierstep (glacier/wgsl/glacierstep.wgsl).
template <int NL>
__device__ __forceinline__ void b_land_surface(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const float DS = P.deltsec;
  // Every input is read before the first store (the compiler cannot prove
  // the fields distinct, so a store would order each later load after it).
  // Each output is formed in registers and stored once, with the value of
  // the shaders' last store to it.
  const float dls = F.dls[c], dglac = F.dglac[c];
  const bool land = dls > 0.f;
  const bool wetsoil = K.NWETSOIL != 0.f && dls > 0.5f;
  const bool veg = K.NVEG > 0.f && land && dglac < 0.90f;
  const bool glacier = dglac > 0.5f && land;
  const bool glaciers = K.NGLACIER != 0.f;
  const float dts = F.land_dts[c];
  float albclim = clim14(F.dalbcl, P.surf + 3, c, SN);
  float albclim1 = clim14(F.dalbcl1, P.surf + 3, c, SN);
  float albclim2 = clim14(F.dalbcl2, P.surf + 3, c, SN);
  const float dwater = wetsoil ? F.dwater[c] : 0.f;
  float driver = 0.f, drunoff = 0.f, dp = 0.f, dsnowz = 0.f, dforest = 0.f, dwmax = 0.f, dwatc = 0.f;
  float soil[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  if (land) {
    driver = F.driver[c];
    drunoff = F.drunoff[c];
    dp = F.dp[c];
    dsnowz = F.dsnowz[c];
    dforest = F.dforest[c];
    dwmax = F.dwmax[c];
    dwatc = F.dwatc[c];
#pragma unroll
    for (int i = 0; i < 5; ++i) soil[i] = F.dsoilt[i * SN + c];
  }
  float co2 = 0.f, dq_low = 0.f, dcveg = 0.f, dcsoil = 0.f, dagg = 0.f, dfd = 0.f, devap = 0.f, dgrow = 0.f;
  float dmr = 0.f, dsc = 0.f, z0c = 0.f;
  if (veg) {
    co2 = F.co2[slot];
    dq_low = F.dq[(NL - 1) * SN + c];
    dcveg = F.dcveg[c];
    dcsoil = F.dcsoil[c];
    dagg = F.dagg[c];
    dfd = F.dfd[NL * SN + c];
    devap = F.devap[c];
    dgrow = F.dgrow[c];
    dmr = F.dmr[c];
    dsc = F.dsc[c];
    if (K.NVEG == 2.f) z0c = F.dz0climo[c];
  }
  const float dpersist_in = glaciers ? F.dpersist[c] : 0.f;
  if (wetsoil) {
    if (dts > 273.15f) {
      const float bf = dwater / K.WSMAX;
      const float al = 1.f / 5.2f * fpow(fpow(fmaxf(bf, 1.0e-3f), (1.f - 4.f) / 4.f) - 1.f, 1.f / 4.f);
      const float dry = expf(-powi(bf * 25.f, 6));
      const float wet = expf(-powi((1.f - bf) * 30.f, 9));
      albclim = K.ALBLANDMAX * dry + al * (1.f - dry - wet) + K.DOCEANALB1 * wet;
      albclim1 = albclim;
      albclim2 = K.ALBLANDMAX * dry + al * (1.f - dry - wet) + K.DOCEANALB2 * wet;
    } else {
      albclim = K.ALBLAND;
      albclim1 = K.DGROUNDALB1;
      albclim2 = K.DGROUNDALB2;
    }
  }
  float dalb = 0.f, dsalb1 = 0.f, dsalb2 = 0.f, drhs = 0.f, dqs = 0.f;
  bool put_alb = false, put_rhs = false;
  if (land) {
    dqs = K.RDBRV * K.RA1 * expf(K.RA2 * (dts - K.TMELT) / (dts - K.RA4)) / dp;
    dqs = dqs / (1.f - (1.f / K.RDBRV - 1.f) * dqs);
    const float dsnow = dsnowz;
    if (dsnow > 0.f) {
      const float forest = dforest;
      auto snow_albedo = [&](float mxf, float mxb, float mnf, float mnb) {
        const float zmax = forest * mxf + (1.f - forest) * mxb;
        const float zmin = forest * mnf + (1.f - forest) * mnb;
        const float zd = (zmax - zmin) * (dts - 263.16f) / (K.TMELT - 263.16f);
        return fmaxf(zmin, fminf(zmax, zmax - zd));
      };
      const float s0 = snow_albedo(K.ALBSMAXF, K.ALBSMAX, K.ALBSMINF, K.ALBSMIN);
      const float s1 = snow_albedo(K.ALBSMAXF1, K.ALBSMAX1, K.ALBSMINF1, K.ALBSMIN1);
      const float s2 = snow_albedo(K.ALBSMAXF2, K.ALBSMAX2, K.ALBSMINF2, K.ALBSMIN2);
      dalb = albclim + (s0 - albclim) * dsnow / (dsnow + 0.01f);
      dsalb1 = albclim1 + (s1 - albclim1) * dsnow / (dsnow + 0.01f);
      dsalb2 = albclim2 + (s2 - albclim2) * dsnow / (dsnow + 0.01f);
      drhs = 1.f;
      put_rhs = true;
    } else {
      dalb = albclim;
      dsalb1 = albclim1;
      dsalb2 = albclim2;
      if (dwmax > 0.f) {
        drhs = fminf(1.f, dwatc / (K.DRHSFULL * dwmax));
        put_rhs = true;
      }
    }
    put_alb = true;
  }
  float npp = 0.f, cveg = 0.f, csoil = 0.f, vsoil = 0.f, lai = 0.f, dz0 = 0.f, wmax = 0.f, forest = 0.f;
  if (veg) {
    float zbeta = 0.f;
    if (!(co2 < 1.0e-8f)) zbeta = fmaxf(0.f, 1.f + K.CO2_SENS * logf((co2 - K.CO2_COMP) / (K.CO2_REF - K.CO2_COMP)));
    const float ts = dts, dsnow = dsnowz;
    float zwmax = dwmax;
    const float zglacfree = 1.f - dglac;
    const float zsvp = K.RA1 * expf(K.RA2 * (ts - K.TMELT) / (ts - K.RA4));
    const float zvpd = fmaxf(0.01f, zsvp - dp * dq_low / 0.622f);
    cveg = dcveg;
    csoil = dcsoil;
    const float zlaim = K.ZLAIMIN + 0.63661977236758f * K.ZLAIMAX * atanf(K.CVEG_L * 2.f * dagg * cveg);
    const float zvegm = 1.f - expf(-K.CVEG_K * zlaim);
    float zveg = 0.f;
    if (zwmax > 0.f) zveg = fminf(fminf(1.f, zvegm), fmaxf(0.f, dwatc / (zwmax * K.VWS_CRIT)));
    const float zft = fminf(1.f, fmaxf(0.f, (ts - K.TMELT) / K.CT_CRIT));
    const float zgppl = K.RLUE * zbeta * zft * zveg * dfd;
    float zgppw = 0.f;
    if (!(co2 < 1.0e-8f)) zgppw = K.CO2CONV * dp * zveg * (-devap) / zvpd * (0.3f * co2);
    zgppw = fminf(1.f, fmaxf(0.f, zgppw));
    const float zgpp = fminf(zgppl, zgppw);
    npp = dgrow * 0.5f * zgpp * zglacfree;
    const float zlitter = cveg / K.TAU_VEG;
    const float zres = fpow(K.Q10, (ts - K.TMELT - 10.f) / 10.f) * csoil / K.TAU_SOIL;
    cveg = cveg + (npp - zlitter) * DS * K.NCVEG;
    csoil = csoil + (zlitter - zres) * DS * K.NCVEG;
    const float zforest = fminf(1.f, fmaxf(0.f, (atanf(cveg - K.CVEG_A) - K.CVEG_E) / (K.CVEG_C - K.CVEG_E)));
    vsoil = fminf(1.f, fmaxf(0.f, (atanf(cveg - K.CVEG_F) - K.CVEG_G) / (K.CVEG_C - K.CVEG_G)));
    lai = -logf(1.f - zveg) / K.CVEG_K;
    const float zvz0 = dmr * zforest + K.VZ0_MIN * (1.f - zforest);
    float zvalb = K.VALB_MIN * zveg + K.VALB_MAX * (1.f - zveg);
    zwmax = K.VWMAX_MAX * vsoil + K.VWMAX_MIN * (1.f - vsoil);
    float zvrhs = dsc * fminf(1.f, fmaxf(0.f, dwatc / (zwmax * K.VWS_CRIT)));
    if (dsnow > 0.f) {
      float zalbsn = (K.ALBSMAX - K.ALBSMIN) * (ts - 263.16f) / (K.TMELT - 263.16f);
      zalbsn = fmaxf(K.ALBSMIN, fminf(K.ALBSMAX, K.ALBSMAX - zalbsn));
      zvalb = zvalb + (zalbsn - zvalb) * dsnow / (dsnow + 0.01f);
      zvalb = K.VSALB_MIN * zforest + zvalb * (1.f - zforest);
      zvrhs = 1.f;
    }
    if (K.NVEG == 2.f) {
      dz0 = sqrtf(zvz0 * zvz0 + z0c * z0c);
      wmax = zwmax;
      drhs = zvrhs;
      put_rhs = true;
      dalb = zvalb;
      forest = zforest;
    }
  }
  if (glacier) {
    auto glacier_albedo = [&](float mx, float mn) {
      return fmaxf(mn, fminf(mx, mx - (mx - mn) * (dts - 263.16f) / (K.TMELT - 263.16f)));
    };
    dalb = glacier_albedo(K.ALBGMAX, K.ALBGMIN);
    dsalb1 = glacier_albedo(K.ALBGMAX1, K.ALBGMIN1);
    dsalb2 = glacier_albedo(K.ALBGMAX2, K.ALBGMIN2);
    drhs = 1.f;
    put_rhs = true;
  }
  float dpersist = dpersist_in, glac = dglac;
  bool put_persist = false, put_glac = false;
  if (glaciers) {
    const bool lnd = dls > 0.5f;
    if (lnd && dsnowz < K.GLACELIM) {
      dpersist = 0.f;
      put_persist = true;
    }
    if (lnd && dsnowz < 0.1f) {
      glac = 0.f;
      put_glac = true;
    }
    if (P.surf[6] > 0.5f) {
      if (dpersist > 0.5f) {
        glac = 1.f;
        put_glac = true;
      }
      dpersist = dls >= 0.5f ? 1.f : 0.f;
      put_persist = true;
    }
  }
  F.dalbclim[c] = albclim;
  F.dalbclim1[c] = albclim1;
  F.dalbclim2[c] = albclim2;
  if (land) {
    F.driver[c] = driver + drunoff * DS;
    F.land_dtsm[c] = dts;
    F.land_dqs[c] = dqs;
    F.dsnow[c] = dsnowz;
    F.dtsoil[c] = soil[0];
    F.dtd2[c] = soil[1];
    F.dtd3[c] = soil[2];
    F.dtd4[c] = soil[3];
    F.dtd5[c] = soil[4];
    F.dt[NL * SN + c] = dts;
    F.dq[NL * SN + c] = dqs;
  }
  if (put_alb) {  // land: the land pass wrote all three albedos, and glaciers lie on land
    F.dalb[c] = dalb;
    F.dsalb[c] = dsalb1;
    F.dsalb[SN + c] = dsalb2;
  }
  if (put_rhs) F.drhs[c] = drhs;
  if (veg) {
    F.dnpp[c] = npp;
    F.dcveg[c] = cveg;
    F.dcsoil[c] = csoil;
    F.dvsoil[c] = vsoil;
    F.dlai[c] = lai;
    if (K.NVEG == 2.f) {
      F.dz0[c] = dz0;
      F.dwmax[c] = wmax;
      F.dforest[c] = forest;
    }
  }
  if (put_persist) F.dpersist[c] = dpersist;
  if (put_glac) F.dglac[c] = glac;
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_land_surface(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_land_surface<NL>(m, pcr, tabr);
}


// seastep coupling and icestep up to getiflx (physics/sea-ice/wgsl/ice.wgsl).
template <int NL>
__device__ __forceinline__ void b_sea_ice(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  if (P.coupled == 0.f) return;
  const bool sea = F.dls[c] < 0.5f;
  float xheat = 0.f, xprs = 0.f;
  if (sea) {
    const float naccua = F.sea_naccua[c] + 1.f;
    xheat = (F.dshfl[c] + F.dswfl[NL * SN + c] + F.dlwfl[NL * SN + c] + F.dlhfl[c] + F.sea_cheata[c]) / naccua;
    xprs = (F.dprs[c] + F.sea_cprsa[c]) / naccua;
  }
  // Every input is read before the first store (the compiler cannot prove
  // the fields distinct); the stores come at the end.
  const float zrhoilfdt = K.CRHOI * K.CLFI / K.XDT;
  const float clssto = clim14(F.xclsst, P.surf, c, SN);
  const float clsst2 = clim14(F.xclsst, P.surf + 3, c, SN);
  const float cliced = fmaxf(clim14(F.xcliced, P.surf + 3, c, SN), 0.f);
  float clicec = fmaxf(clim14(F.xclicec, P.surf + 3, c, SN), 0.f);
  if (cliced <= 0.f) clicec = 0.f;
  const float xls = F.xls[c], xsst = F.xsst[c];
  float xiced = F.xiced[c], xsnow = F.xsnow[c], xicecc = F.xicecc[c], xcflux = F.xcflux[c], xcfluxf = F.xcfluxf[c];
  const float snow_old = xsnow, xicec_in = F.xicec[c], xoflux = F.xoflux[c], zflx_in = F.ice_zflx[c];
  const float xgw = F.xgw[c];
  const float zicedold = xls < 0.5f ? xiced : 0.f;
  float ximelt = 0.f, xsmelt = 0.f, xsmflx = 0.f, xscflx = 0.f, xsndch = 0.f, xcfluxr = 0.f;
  if (xicec_in >= K.CICEMIN) {
    xsnow = xsnow + xprs * K.XDT;
    xprs = 0.f;
  }
  float xts = F.xts[c], xqmelt = 0.f;
  const float ztso = fminf(K.TMELT, xts);
  const float zhsnow = 1.0e3f / K.CRHOSN * xsnow;
  if (xiced >= K.XMIND) {
    const float zcpdt = K.XMIND * K.CRHOI * K.CPI / K.XDT;
    const float zckap = (K.CKAPSN * zhsnow + K.CKAPI * xiced) / (zhsnow + xiced);
    float zkapz = zckap / (xiced + zhsnow);
    if (xiced >= K.XMAXD && K.XMAXD >= 0.f) zkapz = 0.f;
    const float zflx = xheat + zkapz * xsst;
    xts = (zcpdt * ztso + zflx) / (zcpdt + zkapz);
    if (xts > K.TMELT) {
      xqmelt = xheat + zkapz * (xsst - K.TMELT) - zcpdt * (K.TMELT - ztso);
      xts = K.TMELT;
    }
  } else {
    xts = xsst;
    if (xiced > 0.f) xqmelt = xheat;
  }
  if (xiced < K.XMIND) {
    xcflux = xheat;
    xcfluxf = 0.f;
  } else {
    const float zhsnowc = 1.0e3f / K.CRHOSN * xsnow;
    float zckap = (K.CKAPSN * zhsnowc + K.CKAPI * xiced) / (zhsnowc + xiced);
    if (K.XMAXD >= 0.f && xiced >= K.XMAXD) zckap = 0.f;
    xcflux = zckap * (xts - xsst) / (zhsnowc + xiced);
    xcfluxf = zckap * (K.TFREEZE - xsst) / (zhsnowc + xiced);
  }
  if (xicec_in < K.CICEMIN && xprs > 0.f) {
    xcflux = xcflux - xprs * 1000.f * K.CLFSN;
    xsmelt = xprs + xsmelt;
    xsmflx = xsmflx + xprs * 1000.f * K.CLFSN;
    xprs = 0.f;
  }
  float zqmelt = xqmelt;
  if (xiced > 0.f) {
    if (xqmelt > xsnow * 1000.f * K.CLFSN / K.XDT) {
      xsmelt = xsmelt + xsnow / K.XDT;
      xsmflx = xsmflx + xsnow * 1000.f * K.CLFSN / K.XDT;
      zqmelt = xqmelt - xsnow * 1000.f * K.CLFSN / K.XDT;
      xsnow = 0.f;
    } else if (xqmelt > 0.f && xsnow > 0.f) {
      xsmelt = xsmelt + xqmelt / K.CLFSN / 1000.f;
      xsnow = xsnow - xqmelt * K.XDT / K.CLFSN / 1000.f;
      xsmflx = xsmflx + xqmelt;
      zqmelt = 0.f;
    }
    xcflux = xcflux + zqmelt;
  } else {
    xsmelt = xsmelt + xsnow / K.XDT;
    xcflux = xcflux - xsnow * 1000.f * K.CLFSN / K.XDT;
    xsmflx = xsmflx + xsnow * 1000.f * K.CLFSN / K.XDT;
    xsnow = 0.f;
  }
  if (xls < 0.5f && 1.0e3f * xsnow > (K.CRHOS - K.CRHOI) * xiced) {
    const float zhice = (1.0e3f * xsnow + K.CRHOI * xiced) / K.CRHOS;
    const float zdice = zhice - xiced;
    const float zdsnow = -zdice * K.CRHOI / 1.0e3f;
    xsnow = xsnow + zdsnow;
    xscflx = zdsnow * 1.0e3f * K.CLFSN / K.XDT;
    xsmelt = xsmelt - zdsnow / K.XDT;
    xsmflx = xsmflx - zdsnow * 1.0e3f * K.CLFSN / K.XDT;
  }
  if (xls < 0.5f) xcflux = xcflux + xoflux;
  if (xsst <= K.TFREEZE || xiced > 0.f) {
    ximelt = xcflux + xscflx - xcfluxf;
    xiced = xiced - ximelt / zrhoilfdt;
    xcflux = xcfluxf;
  }
  if (xiced <= 0.f) {
    xcflux = xcflux - xiced * zrhoilfdt;
    ximelt = ximelt + xiced * zrhoilfdt;
    xiced = 0.f;
  }
  if (fabsf(xiced) < 1.0e-9f) xiced = 0.f;
  if (xiced > zicedold) xicecc = fminf(xicecc + (1.f - xicecc) * (xiced - zicedold) / 0.5f, 1.f);
  if (xiced < zicedold) xicecc = fmaxf(xicecc + xicecc * (xiced - zicedold) / (2.f * zicedold), 0.f);
  if (xiced <= 0.f) xicecc = 0.f;
  if (K.XMAXD >= 0.f && xiced > K.XMAXD) {
    const float zcflux = (xiced - K.XMAXD) * zrhoilfdt;
    xiced = K.XMAXD;
    xcfluxr = xcfluxr + zcflux;
    ximelt = ximelt + zcflux;
    xsndch = xsndch + zcflux * 1000.f / K.CRHOI / zrhoilfdt;
  }
  float zflx = zflx_in;
  if (xls < 1.f) zflx = fmaxf(0.f, K.XMAXD - xiced) * zrhoilfdt;
  F.sea_cheata[c] = 0.f;
  F.sea_cprsa[c] = 0.f;
  F.sea_naccua[c] = 0.f;
  F.xclssto[c] = clssto;
  F.xclsst2[c] = clsst2;
  F.xcliced2[c] = cliced;
  F.xclicec2[c] = clicec;
  F.ice_snowold[c] = snow_old;
  F.xts[c] = xts;
  F.xqmelt[c] = xqmelt;
  F.ice_zflx[c] = zflx;
  F.ice_part1[c] = xls < 1.f ? xcfluxr * xgw : 0.f;
  F.ice_part2[c] = xls < 1.f ? zflx * xgw : 0.f;
  F.xiced[c] = xiced;
  F.xsnow[c] = xsnow;
  F.xicecc[c] = xicecc;
  F.xicec[c] = xicecc;
  F.xcflux[c] = xcflux;
  F.xcfluxf[c] = xcfluxf;
  F.xcfluxr[c] = xcfluxr;
  F.ximelt[c] = ximelt;
  F.xsmelt[c] = xsmelt;
  F.xsmflx[c] = xsmflx;
  F.xsndch[c] = xsndch;
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_sea_ice(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_sea_ice<NL>(m, pcr, tabr);
}


// seastep (physics/sea/wgsl/seastep.wgsl) with ice_finish (sea-ice/wgsl/finish.wgsl)
// and oceanstep (ocean/wgsl/oceanstep.wgsl).
template <int NL>
__device__ __forceinline__ void b_sea(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const bool coupled = P.coupled != 0.f;
  // Every input is read before the first store (the compiler cannot prove
  // the fields distinct, so a store would order each later load after it);
  // the values this column stores and reads again stay in registers.
  const float dls = F.dls[c];
  const bool open = dls < 0.5f;  // the atmosphere's sea column
  float xls = 0.f, xcflux = 0.f, xcfluxr = 0.f, zflx_in = 0.f, xiced = 0.f, xicec_in = 0.f, xsnow = 0.f;
  float xsmelt = 0.f, xsmflx = 0.f, yclsst2 = 0.f, yls = 0.f, ymld = 0.f, yfldo = 0.f, ysst = 0.f, xsndch = 0.f;
  float snow_old = 0.f, naccua = 0.f;
  if (coupled) {
    xls = F.xls[c];
    xcflux = F.xcflux[c];
    xcfluxr = F.xcfluxr[c];
    zflx_in = F.ice_zflx[c];
    xiced = F.xiced[c];
    xicec_in = F.xicec[c];
    xsnow = F.xsnow[c];
    xsmelt = F.xsmelt[c];
    xsmflx = F.xsmflx[c];
    yclsst2 = clim14(F.yclsst, P.surf + 3, c, SN);
    yls = F.yls[c];
    ymld = F.ymld[c];
    yfldo = F.yfldo[c];
    ysst = F.ysst[c];
    xsndch = F.xsndch[c];
    snow_old = F.ice_snowold[c];
  } else {
    naccua = F.sea_naccua[c];
  }
  float dts = 0.f, dicec = 0.f, dp = 0.f, taux = 0.f, tauy = 0.f, heat_sum = 0.f, cprsa = 0.f;
  if (open) {
    dts = F.xts[c];
    dp = F.dp[c];
    taux = F.dtaux[c];
    tauy = F.dtauy[c];
    if (!coupled) {
      dicec = F.xicec[c];
      heat_sum = F.dshfl[c] + F.dswfl[NL * SN + c] + F.dlwfl[NL * SN + c] + F.dlhfl[c] + F.sea_cheata[c];
      cprsa = F.dprs[c] + F.sea_cprsa[c];
    }
  }
  float zsst = 0.f;
  if (coupled) {
    const double s1 = m.sums[slot * 4 + 2], s2 = m.sums[slot * 4 + 3];
    if (s1 > 0.0 && s2 > 0.0 && xls < 1.f) {
      float zflx = zflx_in;
      const float zfac = (float)(s1 / s2);
      if (zfac <= 1.f) zflx = zflx * zfac;
      xcfluxr = xcfluxr - zflx;
      xcflux = xcflux - zflx;
    }
    const float xicec = xicec_in >= K.THICEC ? 1.f : 0.f;
    const bool melt = xiced <= 0.f && xsnow > 0.f;
    if (melt) {
      const float zcflux = xsnow * 1000.f * K.CLFSN / K.XDT;
      xsmelt = xsmelt + xsnow / K.XDT;
      xsmflx = xsmflx + zcflux;
      xcflux = xcflux - zcflux;
      xsnow = 0.f;
    }
    const bool sea = xls < 0.5f;
    const float heat = sea ? xcflux : 0.f;
    const float yiced = xiced;
    const float zcpsdt = K.DTMIX / (K.CRHOS * K.CPS);
    float yiflux = 0.f;
    zsst = ysst;
    if (yls < 1.f && yiced <= 0.f) zsst = zsst + (heat + yfldo) * zcpsdt / ymld;
    if (yls < 1.f && yiced > 0.f) yiflux = yiflux - yfldo - heat;
    if (ysst < K.TFREEZE && yls < 1.f) {
      yiflux = yiflux + (K.TFREEZE - zsst) * ymld / zcpsdt;
      zsst = K.TFREEZE;
    }
    if (yiced > 0.f && yls < 1.f) {
      const float zf = (K.TFREEZE - zsst) * ymld / zcpsdt;
      zsst = zsst + zf * zcpsdt / ymld;
      yiflux = yiflux + zf;
    }
    if (sea) xsndch = xsndch + (xsnow - snow_old);
    F.xcfluxr[c] = xcfluxr;
    if (melt) F.xsmflx[c] = xsmflx;
    F.xicec[c] = xicec;
    F.xsnow[c] = xsnow;
    F.xsmelt[c] = xsmelt;
    F.xcflux[c] = xcflux;
    F.yclsst2[c] = yclsst2;
    F.ysst[c] = zsst;
    F.xsst[c] = zsst;
    F.xmld[c] = ymld;
    F.xoheat[c] = -yiflux;
    F.xoflux[c] = -yiflux;
    if (sea) F.xsndch[c] = xsndch;
    dicec = xicec;
  } else {
    F.sea_naccua[c] = naccua + 1.f;
  }
  if (!open) return;
  if (coupled) {
    F.sea_dsst[c] = zsst;
    F.sea_dts[c] = dts;
    F.dmld[c] = ymld;
    F.dicec[c] = dicec;
    F.diced[c] = xiced;
    F.dsnow[c] = xsnow;
    F.dsmelt[c] = xsmelt;
    F.dsndch[c] = xsndch;
  } else {
    F.sea_cheata[c] = heat_sum;
    F.sea_cprsa[c] = cprsa;
  }
  F.dt[NL * SN + c] = dts;
  float dqs = K.RDBRV * K.RA1 * expf(K.RA2 * (dts - K.TMELT) / (dts - K.RA4)) / dp;
  dqs = dqs / (1.f - (1.f / K.RDBRV - 1.f) * dqs);
  F.sea_dqs[c] = dqs;
  F.dq[NL * SN + c] = dqs;
  // The stress magnitude's sum of squares is one explicit fused multiply-add,
  // so that its rounding does not depend on where the loads above are placed.
  const float zz0 = fmaxf(K.CHARNOCK * sqrtf(__fmaf_rn(taux, taux, tauy * tauy)) * K.GASCON * dts / (K.GA * dp), K.DZ0SEA);
  F.drhs[c] = K.DRHSSEA * (1.f - dicec) + K.DRHSICE * dicec;
  F.dalb[c] = K.ALBSEA * (1.f - dicec) + dicec * fminf(K.ALBICE, 0.5f + 0.025f * (273.f - dts));
  F.dsalb[c] = K.DOCEANALB1 * (1.f - dicec) + dicec * fminf(K.DICEALBMX1, K.DICEALBMN1 + 0.025f * (273.f - dts));
  F.dsalb[SN + c] = K.DOCEANALB2 * (1.f - dicec) + dicec * fminf(K.DICEALBMX2, K.DICEALBMN2 + 0.025f * (273.f - dts));
  F.dz0[c] = zz0 * (1.f - dicec) + K.DZ0ICE * dicec;
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_sea(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_sea<NL>(m, pcr, tabr);
}


// carbonstep (physics/carbon/wgsl/carbonstep.wgsl).
template <int NL>
__device__ __forceinline__ void b_carbon(const Model& m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  // inputs first: the compiler cannot prove the fields distinct
  const float precip = (F.dprc[c] + F.dprl[c]) * 3.154e9f;
  const float avgprecip = F.localavgprecip[c];
  const bool carbon = P.carbon != 0.f;
  const float tsurf = carbon ? F.dt[NL * SN + c] : 0.f;
  const float dls = carbon ? F.dls[c] : 0.f, co2 = carbon ? F.co2[slot] : 0.f, dp = carbon ? F.dp[c] : 0.f;
  const float avgtemps = carbon ? F.localavgtemps[c] : 0.f, avgweather = carbon ? F.localavgweather[c] : 0.f;
  float local_weathering = carbon ? F.localweathering[c] : 0.f;
  F.localprecip[c] = precip;
  F.localavgprecip[c] = avgprecip + precip * K.TIMEWEIGHT;
  if (!carbon) return;
  if (K.NCARBON != 0.f) {
    float weathering = 0.f;
    if (dls > 0.5f && tsurf >= 273.15f) {
      const float pco2 = co2 * dp * 1.0e-5f;
      weathering = fpow(pco2 / K.CO2EARTH, K.BETA) * expf(K.KACT * (tsurf - 288.f)) * fpow(precip / K.PEARTH, 0.65f);
      if (K.NSUPPLY != 0.f) {
        const float wmaxp = fmaxf(K.WMAX / K.VEARTH, 2.0e-15f);
        weathering = wmaxp * (1.f - expf(-weathering / wmaxp));
      }
    }
    local_weathering = weathering * (K.PLARAD * K.PLARAD) / (K.RAD_EARTHSQ * 0.29f);
    F.localweathering[c] = local_weathering;
  }
  F.localavgtemps[c] = avgtemps + tsurf * K.TIMEWEIGHT;
  F.localavgweather[c] = avgweather + local_weathering * K.TIMEWEIGHT;
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_carbon(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  b_carbon<NL>(m, pcr, tabr);
}


// snapshot/wgsl/pack.wgsl: the published fields, window extrema, RH.
template <int NL>
__global__ void __launch_bounds__(kBlock) k_pack(Model m, const PlanetConst* __restrict__ pcr, const float* __restrict__ tabr) {
  COLUMN_PROLOGUE
  const int step = (int)P.snap[0], window = (int)P.snap[1];
  const float t = F.dt[NL * SN + c];
  float* tr = F.snapshot_tracking + c;
  if (tr[7 * SN] == 0.f) {
    tr[0] = t;
    tr[SN] = t;
    tr[7 * SN] = 1.f;
  }
  tr[0] = fminf(tr[0], t);
  tr[SN] = fmaxf(tr[SN], t);
  if (step > 0 && window > 0 && step % window == 0) {
    const float range = tr[SN] - tr[0];
    tr[2 * SN] = tr[0];
    tr[3 * SN] = tr[SN];
    tr[4 * SN] = range;
    tr[5 * SN] += range;
    tr[6 * SN] += 1.f;
    tr[7 * SN] = 0.f;
    tr[8 * SN] = 1.f;
  }
  // The pack itself writes the publishing step's snapshot (snap[2] = 1).
  // F.dca_skip and the scratch slots are not published.
  float* S = F.snapshot + c;
  auto put = [&](int index, float v) { S[(size_t)index * SN] = v; };
  const float snapflag = P.snap[2];
  if (h == 0) {
    // The step's CPU values, kept in their state slots for checkpoints.
    for (int i = 0; i < 3; ++i) F.snapshot_step[i * d.S + slot] = P.snap[i];
    for (int i = 0; i < 5; ++i) F.radiation_step[i * d.S + slot] = P.rad[i];
    for (int i = 0; i < 7; ++i) F.surface_step[i * d.S + slot] = P.surf[i];
    F.carbon_step[slot] = P.carbon;
  }
  if (snapflag == 0.f) return;
  const int jet = (int)K.JET;
  put(0, F.dt[NL * SN + c]);
  put(1, F.dtsa[c]);
  put(2, F.du[(NL - 1) * SN + c]);
  put(3, F.dv[(NL - 1) * SN + c]);
  put(4, F.dcc[NL * SN + c]);
  put(5, F.dprc[c] + F.dprl[c]);
  put(6, F.dp[c]);
  put(7, F.dqvi[c]);
  put(8, F.dicec[c]);
  put(9, F.dsnow[c]);
  put(10, F.dwatc[c]);
  put(11, F.dalb[c]);
  put(12, F.du[jet * SN + c]);
  put(13, F.dv[jet * SN + c]);
  put(14, -F.dlwfl[c]);
  put(15, F.dls[c]);
  put(16, F.dswfl[c] + F.dlwfl[c]);
  put(17, F.dsmelt[c] * -333700000.f + F.dswfl[NL * SN + c] + F.dlwfl[NL * SN + c] + F.dshfl[c] + F.dlhfl[c]);
  put(18, -F.devap[c]);
  put(19, F.drunoff[c]);
  put(20, F.dforest[c]);
  put(21, F.dlai[c]);
  put(22, F.dprs[c]);
  put(23, F.dsmelt[c]);
  put(24, F.diced[c]);
  put(25, F.dglac[c]);
  put(27, F.dswfl[NL * SN + c]);
  put(28, F.dlwfl[NL * SN + c]);
  put(29, F.dshfl[c]);
  put(30, F.dlhfl[c]);
  put(31, F.dprc[c]);
  put(32, F.dprl[c]);
  put(33, F.dswfl[c]);
  put(34, F.dlwfl[c]);
  const bool windowed = tr[8 * SN] != 0.f;
  put(35, windowed ? tr[2 * SN] : tr[0]);
  put(36, windowed ? tr[3 * SN] : tr[SN]);
  put(37, windowed ? tr[4 * SN] : tr[SN] - tr[0]);
  put(38, tr[5 * SN]);
  put(39, tr[6 * SN]);
  put(40, F.dnpp[c]);
  put(41, F.gmu0[c]);
  tr[5 * SN] = 0.f;
  tr[6 * SN] = 0.f;
#pragma unroll
  for (int l = 0; l < NL; ++l) {
    const int f = 51 + 5 * l;
    put(f, F.dt[l * SN + c]);
    put(f + 1, F.du[l * SN + c]);
    put(f + 2, F.dv[l * SN + c]);
    put(f + 4, F.dcc[l * SN + c]);
  }
  put(42, F.capen[c]);
  put(43, F.lnb[c]);
  put(44, F.mpoti[c]);
  put(45, F.chim[c]);
  put(46, F.laav[c]);
  put(47, F.venti[c]);
  put(48, F.vrmpi[c]);
  put(49, F.gpi[c]);
  put(50, F.shear[c]);
  const int lowest = NL - 1;
  const float qsat = sat_divided(K, F.dt[lowest * SN + c], F.dp[c] * K.SIGMA_LOW);
  put(51 + 5 * lowest + 3, fmaxf(0.f, F.dq[lowest * SN + c]) / fmaxf(1.17549435e-38f, qsat));
}

// Non-finite check per slot over the prognostic spectral state: sets
// flags[slot] = 1 when any coefficient of sp, st, sz, sd or sq is NaN or Inf.
__global__ void k_finite(Model m) {
  const Dims& d = m.d;
  const int SR = d.S * d.NRSP;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= SR) return;
  const int slot = c / d.NRSP;
  if (!m.params[slot].active) return;
  const int l = blockIdx.y;
  const size_t i = (size_t)l * SR + c;
  const float v = m.f.st[i] + m.f.sz[i] + m.f.sd[i] + m.f.sq[i] + (l == 0 ? m.f.sp[c] : 0.f);
  if (!isfinite(v)) m.flags[slot] = 1;
}



// Fused column kernels (each thread takes its column through consecutive
// routines in the reference's order, stepper/index.ts:148-161): kuo + mkdca,
// rain + soil, land surface + sea ice, sea + carbon. A routine re-reads what
// the one before it wrote or read for the same column from L1/L2 instead of
// HBM. The full step uses the two that measured faster than their parts
// (see phy_fused_precipitation_to_carbon); stage replay (exogcm_run_stage)
// runs the separate kernels, and a full step equals its stages bit for bit.
template <int NL>
__global__ void __launch_bounds__(kBlock, 4) k_fused_kuo_mkdca(Model m, const PlanetConst* __restrict__ pcr,
                                                               const float* __restrict__ tabr) {
  b_kuo<NL>(m, pcr, tabr);
  b_mkdca<NL>(m, pcr, tabr);
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_fused_rain_soil(Model m, const PlanetConst* pcr, const float* tabr) {
  b_rain_column<NL>(m, pcr, tabr);
  b_soil<NL>(m, pcr, tabr);
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_fused_land_seaice(Model m, const PlanetConst* __restrict__ pcr,
                                                              const float* __restrict__ tabr) {
  b_land_surface<NL>(m, pcr, tabr);
  b_sea_ice<NL>(m, pcr, tabr);
}
template <int NL>
__global__ void __launch_bounds__(kBlock) k_fused_sea_carbon(Model m, const PlanetConst* __restrict__ pcr,
                                                             const float* __restrict__ tabr) {
  b_sea<NL>(m, pcr, tabr);
  b_carbon<NL>(m, pcr, tabr);
}


COLUMN_LAUNCHER(FixerColumn, k_fixer_column)
COLUMN_LAUNCHER(FusedKuoMkdca, k_fused_kuo_mkdca)
COLUMN_LAUNCHER(FusedRainSoil, k_fused_rain_soil)
COLUMN_LAUNCHER(FusedLandSeaice, k_fused_land_seaice)
COLUMN_LAUNCHER(FusedSeaCarbon, k_fused_sea_carbon)
template <int NL>
struct Swr {
  static void run(const Model& m, cudaStream_t st) {
    k_swr<NL><<<nblocks((size_t)m.d.S * m.d.NHOR, kBlock / 2), kBlock, 0, st>>>(m);
  }
};
COLUMN_LAUNCHER(LwrRadstep, k_lwr_radstep)
COLUMN_LAUNCHER(Kuo, k_kuo)
COLUMN_LAUNCHER(Mkdca, k_mkdca)
COLUMN_LAUNCHER(RainColumn, k_rain_column)
COLUMN_LAUNCHER(Soil, k_soil)
COLUMN_LAUNCHER(LandSurface, k_land_surface)
COLUMN_LAUNCHER(SeaIce, k_sea_ice)
COLUMN_LAUNCHER(Sea, k_sea)
COLUMN_LAUNCHER(Carbon, k_carbon)
COLUMN_LAUNCHER(Pack, k_pack)

template <int NL>
struct FixerRow {
  static void run(const Model& m, cudaStream_t st) {
    k_fixer_row<NL><<<nblocks((size_t)m.d.S * m.d.NLAT, kRowWarps), 32 * kRowWarps, 0, st>>>(m);
  }
};

}  // namespace

void phy_fixer(const Model& m, cudaStream_t st) {
  by_levels<FixerColumn>(m.d.L, m, st);
  by_levels<FixerRow>(m.d.L, m, st);
  k_slot_sums<<<m.d.S, kSumThreads, 0, st>>>(m, m.f.fixneg, m.f.fixpos, m.f.fixsum, 0);
  phy_fixer_apply(m, st);
}

void phy_radiation(const Model& m, cudaStream_t st) {
  phy_solang_mko3(m, st);
  by_levels<Swr>(m.d.L, m, st);
  by_levels<LwrRadstep>(m.d.L, m, st);
}

void phy_precipitation_columns(const Model& m, cudaStream_t st) {
  by_levels<Kuo>(m.d.L, m, st);
  by_levels<Mkdca>(m.d.L, m, st);
  k_mkdca_limit<<<m.d.S, kSumThreads, 0, st>>>(m);
  by_levels<RainColumn>(m.d.L, m, st);
}

void phy_surface(const Model& m, cudaStream_t st) {
  by_levels<Soil>(m.d.L, m, st);
  k_mkradv<<<nblocks((size_t)m.d.S * m.d.NHOR, kBlock), kBlock, 0, st>>>(m);
  by_levels<LandSurface>(m.d.L, m, st);
  by_levels<SeaIce>(m.d.L, m, st);
  k_slot_sums<<<m.d.S, kSumThreads, 0, st>>>(m, m.f.ice_part1, m.f.ice_part2, m.f.ice_sums, 1);
  by_levels<Sea>(m.d.L, m, st);
}

void phy_carbon(const Model& m, cudaStream_t st) { by_levels<Carbon>(m.d.L, m, st); }

// The full step's physics between physics_in and physics_out. Fusing
// consecutive per-column routines into one kernel was measured per pair at
// 128 T42 L10 planets (CUDA events): land surface + sea ice (86.5 against
// 88.7 us) and sea + carbon (57.7 against 60.2 us) pay and run fused; fixer
// apply + surflx + vdiff + solang/mko3 (375.6 against 354.1 us), kuo + mkdca
// (199.7 against 180.6 us) and rain + soil (274.0 against 259.5 us) lost more
// to the fused kernels' register pressure and lower occupancy than they saved
// in re-reads, and run as separate kernels.
void phy_fused_through_radiation(const Model& m, cudaStream_t st) {
  phy_fixer(m, st);
  phy_surface_flux(m, st);
  phy_radiation(m, st);
}

void phy_fused_precipitation_to_carbon(const Model& m, cudaStream_t st) {
  phy_precipitation_columns(m, st);
  by_levels<Soil>(m.d.L, m, st);
  k_mkradv<<<nblocks((size_t)m.d.S * m.d.NHOR, kBlock), kBlock, 0, st>>>(m);
  by_levels<FusedLandSeaice>(m.d.L, m, st);
  k_slot_sums<<<m.d.S, kSumThreads, 0, st>>>(m, m.f.ice_part1, m.f.ice_part2, m.f.ice_sums, 1);
  by_levels<FusedSeaCarbon>(m.d.L, m, st);
}

void phy_pack(const Model& m, cudaStream_t st) { by_levels<Pack>(m.d.L, m, st); }

void phy_finite_check(const Model& m, cudaStream_t st) {
  const dim3 grid(nblocks((size_t)m.d.S * m.d.NRSP, 256), m.d.NLEV);
  k_finite<<<grid, 256, 0, st>>>(m);
}

bool phy_launch_one(const Model& m, const std::string& kernel, cudaStream_t st) {
  const int L = m.d.L;
  if (phy_flux_launch_one(m, kernel, st))
    return true;
  else if (kernel == "storm") {
    Model on = m;
    on.storm = 1;
    phy_storm(on, st);
  } else if (kernel == "swr")
    by_levels<Swr>(L, m, st);
  else if (kernel == "lwr_radstep")
    by_levels<LwrRadstep>(L, m, st);
  else if (kernel == "kuo")
    by_levels<Kuo>(L, m, st);
  else if (kernel == "mkdca")
    by_levels<Mkdca>(L, m, st);
  else if (kernel == "rain_column")
    by_levels<RainColumn>(L, m, st);
  else if (kernel == "soil")
    by_levels<Soil>(L, m, st);
  else if (kernel == "land_surface")
    by_levels<LandSurface>(L, m, st);
  else if (kernel == "sea_ice")
    by_levels<SeaIce>(L, m, st);
  else if (kernel == "sea")
    by_levels<Sea>(L, m, st);
  else if (kernel == "carbon")
    by_levels<Carbon>(L, m, st);
  else if (kernel == "fused_kuo_mkdca")
    by_levels<FusedKuoMkdca>(L, m, st);
  else if (kernel == "fused_rain_soil")
    by_levels<FusedRainSoil>(L, m, st);
  else if (kernel == "fused_land_seaice")
    by_levels<FusedLandSeaice>(L, m, st);
  else if (kernel == "fused_sea_carbon")
    by_levels<FusedSeaCarbon>(L, m, st);
  else
    return false;
  return true;
}

}  // namespace exogcm
