// Field list of the GCM state arena, in the reference's layout order.
//
// TEST INFRASTRUCTURE (oracle): restates stepper/index.ts:38-50 (fields) with
// each module's fields() (dynamics/index.ts:27-66, physics/*/index.ts,
// snapshot/index.ts:14-24). Shapes: S spectral (NRSP per plane), F fourier
// (NLAT*NFC), G grid (NHOR), T table (count is the element count).
// Counts: L = levels, H = levels + 1, or a literal.
#pragma once
// clang-format off
#define ORACLE_FIELDS(X) \
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
