// The GCM state arena's fields, in the reference's layout order.
//
// This order and these names are the checkpoint format's field index
// (checkpoint/restart/index.ts:11-45 writes every slot in layout order), so
// they follow src/model/climate/gcm/stepper/index.ts:38-50 and each module's
// fields() exactly. Shape: S spectral (NRSP floats per plane), F Fourier
// (NLAT*NFC), G grid (NHOR), T table (count = element count). Count: L levels,
// H levels + 1, P snapshot slots (51 + 5 L), or a literal.
#pragma once
// clang-format off
#define EXOGCM_FIELDS(X) \
  X(sd,S,L) X(st,S,L) X(sz,S,L) X(sq,S,L) X(sdp,S,L) X(stp,S,L) X(szp,S,L) X(sqp,S,L) \
  X(sdt,S,L) X(stt,S,L) X(szt,S,L) X(sqt,S,L) X(sdm,S,L) X(stm,S,L) X(szm,S,L) X(sqm,S,L) \
  X(zdsdp1,S,L) X(zdszp1,S,L) X(zdsdp2,S,L) X(zdszp2,S,L) X(zstt1,S,L) X(zstt2,S,L) X(zsdef,S,L) \
  X(sp,S,1) X(spp,S,1) X(spt,S,1) X(spm,S,1) \
  X(gd,G,L) X(gt,G,L) X(gz,G,L) X(gq,G,L) X(gu,G,L) X(gv,G,L) X(dw,G,L) \
  X(gtn,G,L) X(gqn,G,L) X(guz,G,L) X(gvz,G,L) X(gke,G,L) X(gut,G,L) X(gvt,G,L) X(guq,G,L) X(gvq,G,L) \
  X(zu,G,L) X(zv,G,L) X(zdu,G,L) X(zdv,G,L) X(zdtdt,G,L) X(zdekin,G,L) \
  X(gudt,G,L) X(gvdt,G,L) X(gtdt,G,L) X(gqdt,G,L) \
  X(gp,G,1) X(gpj,G,1) X(gpmt,G,1) X(gvpp,G,1) X(dp0,G,1) X(dp,G,1) \
  X(du0,G,H) X(dv0,G,H) X(dq,G,H) X(du,G,H) X(dv,G,H) X(dt,G,H) \
  X(dudt,G,H) X(dvdt,G,H) X(dtdt,G,H) X(dqdt,G,H) \
  X(fgd,F,L) X(fgt,F,L) X(fgz,F,L) X(fgq,F,L) X(fgu,F,L) X(fgv,F,L) \
  X(fgtn,F,L) X(fgqn,F,L) X(fguz,F,L) X(fgvz,F,L) X(fgke,F,L) X(fgut,F,L) X(fgvt,F,L) X(fguq,F,L) X(fgvq,F,L) \
  X(fzu,F,L) X(fzv,F,L) X(fzdu,F,L) X(fzdv,F,L) X(fzdtdt,F,L) X(fzdekin,F,L) \
  X(fgudt,F,L) X(fgvdt,F,L) X(fgtdt,F,L) X(fgqdt,F,L) \
  X(fgp,F,1) X(fgpj,F,1) X(fgpmt,F,1) X(fgvpp,F,1) \
  X(fixq,G,L) X(fixneg,G,1) X(fixpos,G,1) X(fixsum,T,2) \
  X(dz0,G,1) X(dls,G,1) X(drhs,G,1) X(dwatc,G,1) X(dtsa,G,1) X(dtransh,G,1) X(dtransm,G,1) \
  X(dtaux,G,1) X(dtauy,G,1) X(dust3,G,1) X(dshfl,G,1) X(dshdt,G,1) X(devap,G,1) X(dlhfl,G,1) X(dlhdt,G,1) \
  X(dcc,G,H) X(dql,G,H) X(dfu,G,H) X(dfd,G,H) X(dftu,G,H) X(dftd,G,H) X(dswfl,G,H) X(dlwfl,G,H) X(dflux,G,H) \
  X(dqo3,G,L) X(dqco2,G,L) X(dtdtswr,G,L) X(dtdtlwr,G,L) X(dconv,G,L) \
  X(gmu0,G,1) X(dalb,G,1) X(dicec,G,1) X(dsalb,G,2) X(radiation_step,T,5) \
  X(dqt,G,H) X(fdqt,F,L) \
  X(icclev,G,L) X(dprcl,G,L) X(dprll,G,L) X(dprscl,G,L) X(dprsll,G,L) X(dca_dtdt,G,L) X(dca_dqdt,G,L) \
  X(dprc,G,1) X(dprl,G,1) X(dprs,G,1) X(dqvi,G,1) X(icctot,G,1) X(dca_limited,G,1) X(dca_skip,T,1) \
  X(dforest,G,1) X(dglac,G,1) X(dwmax,G,1) X(drunoff,G,1) X(dsnow,G,1) X(dsmelt,G,1) \
  X(dsndch,G,1) X(dtsoil,G,1) X(dtd2,G,1) X(dtd3,G,1) X(dtd4,G,1) X(dtd5,G,1) X(diced,G,1) X(dmld,G,1) \
  X(surface_step,T,7) \
  X(land_dts,G,1) X(land_dtsm,G,1) X(land_dqs,G,1) X(driver,G,1) X(duroff,G,1) \
  X(dvroff,G,1) X(darea,G,1) X(dsnowt,G,1) X(dsnowz,G,1) X(dwater,G,1) X(dz0climo,G,1) \
  X(dalbclim,G,1) X(dalbclim1,G,1) X(dalbclim2,G,1) X(dsoilt,G,5) \
  X(dalbcl,G,14) X(dalbcl1,G,14) X(dalbcl2,G,14) \
  X(dpersist,G,1) \
  X(dcveg,G,1) X(dcsoil,G,1) X(dlai,G,1) X(dvsoil,G,1) X(dagg,G,1) X(dgrow,G,1) X(dsc,G,1) X(dmr,G,1) X(dnpp,G,1) \
  X(xts,G,1) X(xsst,G,1) X(xmld,G,1) X(xls,G,1) X(xiced,G,1) X(xicec,G,1) X(xsnow,G,1) \
  X(xqmelt,G,1) X(xicecc,G,1) X(xcflux,G,1) X(xcfluxf,G,1) X(xoheat,G,1) X(xoflux,G,1) \
  X(xgw,G,1) X(xclsst2,G,1) X(xclicec2,G,1) X(xcliced2,G,1) X(xclssto,G,1) \
  X(xcfluxr,G,1) X(ximelt,G,1) X(xsmelt,G,1) X(xsmflx,G,1) X(xsndch,G,1) \
  X(ice_zflx,G,1) X(ice_snowold,G,1) X(ice_part1,G,1) X(ice_part2,G,1) \
  X(xclsst,G,14) X(xclicec,G,14) X(xcliced,G,14) X(ice_sums,T,2) \
  X(ysst,G,1) X(ymld,G,1) X(yls,G,1) X(yfldo,G,1) X(yclsst2,G,1) X(yclsst,G,14) \
  X(sea_dts,G,1) X(sea_dqs,G,1) X(sea_dsst,G,1) X(sea_cheata,G,1) X(sea_cprsa,G,1) X(sea_naccua,G,1) \
  X(localprecip,G,1) X(localavgprecip,G,1) X(localweathering,G,1) X(localavgweather,G,1) X(localavgtemps,G,1) \
  X(co2,T,1) X(carbon_step,T,1) \
  X(capen,G,1) X(lnb,G,1) X(mpoti,G,1) X(chim,G,1) X(laav,G,1) X(venti,G,1) X(vrmpi,G,1) X(gpi,G,1) X(shear,G,1) \
  X(snapshot,G,P) X(snapshot_tracking,G,9) X(snapshot_step,T,3)
// clang-format on

// Kernel constants per planet (pumamod and every physics module's *ini
// values), under the reference's WGSL override names
// (src/model/climate/gcm/setup/index.ts:53-375). The timestep-dependent ones
// (DELT, DELT2, DELTSEC, DELTSEC2, FILTER, ICE_COUPLED) are per step instead.
#define EXOGCM_CONSTS(X)                                                                           \
  X(PSURF) X(WW) X(CV) X(CT) X(AKAP) X(RDBRV) X(ADV) X(ACPD) X(GA) X(GASCON) X(PLAVOR) X(PNU)      \
  X(PNU21) X(RA1) X(RA2) X(RA4) X(TMELT) X(ALV) X(ALS) X(MOIST) X(ZUMIN) X(VDIFF_B) X(VDIFF_C)     \
  X(VDIFF_D) X(NDHEAT) X(NFIXED) X(ZRLON) X(ZDAWN) X(OZONE) X(A0O3) X(A1O3) X(ACO3) X(BO3) X(CO3) \
  X(ZCONST) X(GSOL0) X(ZSOLAR1) X(ZSOLAR2) X(ZSOLARS1) X(ZSOLARS2) X(TSWR1) X(TSWR2) X(TSWR3)      \
  X(ZB3) X(ZB4) X(ZB5) X(RCOEFF) X(LN_DIFFUSE_RAYLEIGH) X(NSTARTEMP) X(SBK) X(TH2OC) X(TPOFMT)     \
  X(ZFCO2_ZZF2) X(ZAO30) X(ZCO20) X(ZH2O0A) X(ZH2O0) X(ZAO3C) X(ZACO2C) X(ZAH2OC) X(ZTH2OC)       \
  X(RHBETA) X(NBETA) X(PDEEP) X(PDEEPTH) X(RKSHALLOW) X(GAMMA) X(ZRFAC) X(CLWFAC) X(CLWCRIT1)     \
  X(CLWCRIT2) X(SICECAP) X(SOILCAP) X(SICEDIFF) X(SOILDIFF) X(SNOWCAP) X(SNOWDIFF) X(RHOSNOW)      \
  X(DZTOP) X(DSMAX) X(ALBSMAX) X(ALBSMIN) X(ALBSMAXF) X(ALBSMINF) X(ALBSMAX1) X(ALBSMIN1)          \
  X(ALBSMAXF1) X(ALBSMINF1) X(ALBSMAX2) X(ALBSMIN2) X(ALBSMAXF2) X(ALBSMINF2) X(ALBGMAX) X(ALBGMIN) \
  X(ALBGMAX1) X(ALBGMIN1) X(ALBGMAX2) X(ALBGMIN2) X(DRHSFULL) X(NWETSOIL) X(WSMAX) X(ALBLAND)      \
  X(ALBLANDMAX) X(DGROUNDALB1) X(DGROUNDALB2) X(DOCEANALB1) X(DOCEANALB2) X(NVEG) X(RLUE)          \
  X(CO2CONV) X(TAU_VEG) X(TAU_SOIL) X(VWS_CRIT) X(Q10) X(ZLAIMAX) X(ZLAIMIN) X(VALB_MIN)           \
  X(VALB_MAX) X(VSALB_MIN) X(VWMAX_MAX) X(VWMAX_MIN) X(VZ0_MIN) X(CVEG_A) X(CVEG_C) X(CVEG_F)      \
  X(CVEG_K) X(CVEG_L) X(CT_CRIT) X(CO2_REF) X(CO2_COMP) X(CO2_SENS) X(CVEG_E) X(CVEG_G) X(NCVEG)   \
  X(NGLACIER) X(GLACELIM) X(XDT) X(XMIND) X(XMAXD) X(CICEMIN) X(THICEC) X(TFREEZE) X(CRHOI)        \
  X(CRHOS) X(CRHOSN) X(CPI) X(CKAPI) X(CKAPSN) X(CLFI) X(CLFSN) X(DTMIX) X(CPS) X(CHARNOCK)        \
  X(DZ0SEA) X(DZ0ICE) X(DRHSSEA) X(DRHSICE) X(ALBSEA) X(ALBICE) X(DICEALBMX1) X(DICEALBMX2)        \
  X(DICEALBMN1) X(DICEALBMN2) X(NCARBON) X(NSUPPLY) X(TIMEWEIGHT) X(CO2EARTH) X(BETA) X(KACT)      \
  X(PEARTH) X(WMAX) X(VEARTH) X(PLARAD) X(RAD_EARTHSQ) X(JET) X(SIGMA_LOW) X(NSTORMDIAG) X(CKCD)    \
  X(VITHRESH)

// Per-planet constant tables (dynamics set-up, physics level constants):
// name, element count in terms of L (levels), NRSP, NTRU.
#define EXOGCM_PTABLES(X)                                                                          \
  X(t0, L) X(dsigma, L) X(sigma, L) X(sigmah, L) X(rdsig, L) X(t01s2, L) X(tkp, L) X(damp, L)      \
  X(tdisst, L) X(tdissq, L) X(tdissd, L) X(tdissz, L) X(tfrc, L) X(c, L * L) X(g, L * L)           \
  X(tau, L * L) X(bm1, 4 * NTRU * L * L) X(sop, NRSP) X(srp, L * NRSP) X(sakpp, L * NRSP)          \
  X(flux_sigfac, 1) X(flux_lnsig, 1) X(vdiff_skap, L) X(vdiff_skaph, L) X(vdiff_mixh2, L)           \
  X(vdiff_mixm2, L) X(vdiff_rdsig, L) X(vdiff_sigmah3, L) X(vdiff_kfac, L) X(rad_lnsig, L)          \
  X(lwr_zzf1, L) X(lwr_zzf3, L) X(rcrit, L) X(kuo_zfac, L) X(dsoilz, 5)
