// Reference harness: compiles the reference CPU path (src/propagate-tor-test_tbb.cpp)
// UNMODIFIED, from where it lies in the reference checkout, and exposes its own
// functions through a small C ABI so tests can run the reference arithmetic on
// arbitrary Matriplex arrays.
//
// TEST INFRASTRUCTURE ONLY (oracle). Built by oracle/Makefile into oracle/_ref/;
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
// load it, always as the checker or the timed CPU reference, never as the product.
//
// Build-time knobs (see oracle/Makefile):
//   -Dbsize=B -Dntrks=T -Dnevts=E -Dnlayer=L   the reference's own macros (TBB:15-38);
//                                              ntrks/nevts/nlayer only size the fixture
//   -DP2R_REF_RUNTIME_KFACT                    defines `constexpr` away before the include
//                                              so that kfact (TBB:654) becomes a mutable
//                                              global and Bz can be set at run time.
//
// The std headers the reference includes are included first so that the
// `constexpr` redefinition only reaches the reference's own two constants.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <vector>

#include <tbb/tbb.h>

#ifdef P2R_REF_RUNTIME_KFACT
#define constexpr
#endif
#define main p2r_tbb_ref_main
#include P2R_REF_SRC
#undef main
#ifdef P2R_REF_RUNTIME_KFACT
#undef constexpr
#endif

extern "C" {

int ref_bsize(void) { return bsize; }

int ref_runtime_kfact(void) {
#ifdef P2R_REF_RUNTIME_KFACT
  return 1;
#else
  return 0;
#endif
}

float ref_get_kfact(void) { return kfact; }

// kfact = 100/(-0.299792458*Bz), evaluated in double and rounded to float exactly as
// the reference's constant initialiser (TBB:654) is. Only the runtime-kfact build can
// change it; the unmodified build returns -1 unless Bz is the compiled-in 3.8112 T.
int ref_set_bz(double bz) {
#ifdef P2R_REF_RUNTIME_KFACT
  kfact = 100 / (-0.299792458 * bz);
  return 0;
#else
  return (float)(100 / (-0.299792458 * bz)) == kfact ? 0 : -1;
#endif
}

// One Matriplex block: the reference's own propagateToR (TBB:656-812).
void ref_propagate_block(const void* trk_in, const void* hit, void* trk_out) {
  const MPTRK* in = (const MPTRK*)trk_in;
  const MPHIT* h = (const MPHIT*)hit;
  MPTRK* out = (MPTRK*)trk_out;
  propagateToR(&in->cov, &in->par, &in->q, &h->pos, &out->cov, &out->par);
}

// One Matriplex block: the reference's own KalmanUpdate (TBB:433-642), in place.
void ref_update_block(void* trk, const void* hit) {
  MPTRK* t = (MPTRK*)trk;
  const MPHIT* h = (const MPHIT*)hit;
  KalmanUpdate(&t->cov, &t->par, &h->cov, &h->pos);
}

// One Matriplex block: the reference's unused 3x3 routines (TBB:376-426). inv_out: an MP3x3
// block (9*bsize floats); gain_out: an MP3x6 block (18*bsize floats).
void ref_gain_inv_block(const void* trk, const void* hit, void* inv_out) {
  const MPTRK* t = (const MPTRK*)trk;
  const MPHIT* h = (const MPHIT*)hit;
  KalmanGainInv(&t->cov, &h->cov, (MP3x3*)inv_out);
}

void ref_gain_block(const void* trk, const void* inv, void* gain_out) {
  const MPTRK* t = (const MPTRK*)trk;
  KalmanGain(&t->cov, (const MP3x3*)inv, (MP3x6*)gain_out);
}

// The reference driver loop (TBB:870-926) with run-time sizes. chained=0 is the
// reference's "restart" form (every layer propagates the INPUT block, TBB:894);
// chained=1 carries the output block from layer to layer, as the chained GPU
// variants do (cuda_v4.cu:840-846). Indexing: track block ib + nb*ev (TBB:147-153),
// hit block lay + ib*nlayer + ev*nlayer*nb (TBB:215-217).
void ref_run(const void* trk_v, const void* hit_v, void* out_v, long nev, long nbl, int nlay,
             int niter, int nthr, int chained) {
  const MPTRK* trk = (const MPTRK*)trk_v;
  const MPHIT* hit = (const MPHIT*)hit_v;
  MPTRK* outtrk = (MPTRK*)out_v;
  tbb::global_control c(tbb::global_control::max_allowed_parallelism, size_t(nthr));
  for (int itr = 0; itr < niter; itr++) {
    tbb::parallel_for(tbb::blocked_range<size_t>(0, size_t(nev), 4), [&](tbb::blocked_range<size_t> iex) {
      for (size_t ie = iex.begin(); ie < iex.end(); ++ie) {
        tbb::parallel_for(tbb::blocked_range<size_t>(0, size_t(nbl), 4), [&](tbb::blocked_range<size_t> ibx) {
          for (size_t ib = ibx.begin(); ib < ibx.end(); ++ib) {
            const MPTRK* btracks = &trk[ib + nbl * ie];
            MPTRK* obtracks = &outtrk[ib + nbl * ie];
            (*obtracks) = (*btracks);
            for (size_t layer = 0; layer < size_t(nlay); ++layer) {
              const MPHIT* bhits = &hit[layer + ib * nlay + ie * nlay * nbl];
              if (chained)
                propagateToR(&obtracks->cov, &obtracks->par, &obtracks->q, &bhits->pos, &obtracks->cov,
                             &obtracks->par);
              else
                propagateToR(&btracks->cov, &btracks->par, &btracks->q, &bhits->pos, &obtracks->cov,
                             &obtracks->par);
              KalmanUpdate(&obtracks->cov, &obtracks->par, &bhits->cov, &bhits->pos);
            }
          }
        });
      }
    });
  }
}

// Chained loop over blocks whose lanes have their own layer counts (nlay_lane[b*bsize+it],
// 0..nlay_max). The reference functions always process all bsize lanes, so lanes that
// have run out of layers are restored from a copy after each layer: the arithmetic of
// live lanes is the reference's, masked lanes keep their last state.
void ref_run_masked(const void* trk_v, const void* hit_v, void* out_v, long nblocks, int nlay_max,
                    const int* nlay_lane) {
  const MPTRK* trk = (const MPTRK*)trk_v;
  const MPHIT* hit = (const MPHIT*)hit_v;
  MPTRK* outtrk = (MPTRK*)out_v;
  for (long b = 0; b < nblocks; ++b) {
    MPTRK* ob = &outtrk[b];
    *ob = trk[b];
    for (int layer = 0; layer < nlay_max; ++layer) {
      MPTRK keep = *ob;
      const MPHIT* bh = &hit[layer + (size_t)b * nlay_max];
      propagateToR(&ob->cov, &ob->par, &ob->q, &bh->pos, &ob->cov, &ob->par);
      KalmanUpdate(&ob->cov, &ob->par, &bh->cov, &bh->pos);
      for (int it = 0; it < bsize; ++it) {
        if (layer < nlay_lane[b * bsize + it]) continue;
        for (int ip = 0; ip < 6; ++ip) ob->par.data[it + ip * bsize] = keep.par.data[it + ip * bsize];
        for (int ip = 0; ip < 21; ++ip) ob->cov.data[it + ip * bsize] = keep.cov.data[it + ip * bsize];
      }
    }
  }
}

long ref_fixture_nevts(void) { return nevts; }
long ref_fixture_ntrks(void) { return ntrks; }
long ref_fixture_nb(void) { return nb; }
int ref_fixture_nlayer(void) { return nlayer; }

// The reference's own input generation (prepareTracks / prepareHits, TBB:243-293) from
// the fixture src/input_track.h, with the hits listed in the order main uses
// (TBB:818-820). glibc rand() is re-seeded with its default seed (1) first, so each call
// reproduces the sequence a fresh run of the reference program sees.
void ref_prepare_fixture(void* trk_out, void* hit_out) {
#include "input_track.h"
  std::vector<AHIT> inputhits{inputhit21, inputhit20, inputhit19, inputhit18, inputhit17, inputhit16,
                              inputhit15, inputhit14, inputhit13, inputhit12, inputhit11, inputhit10,
                              inputhit09, inputhit08, inputhit07, inputhit06, inputhit05, inputhit04,
                              inputhit03, inputhit02, inputhit01, inputhit00};
  srand(1);
  MPTRK* t = prepareTracks(inputtrk);
  MPHIT* h = prepareHits(inputhits);
  std::memcpy(trk_out, t, sizeof(MPTRK) * nevts * nb);
  std::memcpy(hit_out, h, sizeof(MPHIT) * nevts * nb * nlayer);
  free(t);
  free(h);
}

// Fixture seed track and hits as plain arrays: par[6], cov[21], q, then 22 hits of
// pos[3], cov[6] in the reversed order main uses (TBB:818-820).
void ref_fixture_raw(float* par6, float* cov21, int* q, float* hits22x9) {
#include "input_track.h"
  std::vector<AHIT> inputhits{inputhit21, inputhit20, inputhit19, inputhit18, inputhit17, inputhit16,
                              inputhit15, inputhit14, inputhit13, inputhit12, inputhit11, inputhit10,
                              inputhit09, inputhit08, inputhit07, inputhit06, inputhit05, inputhit04,
                              inputhit03, inputhit02, inputhit01, inputhit00};
  for (int i = 0; i < 6; ++i) par6[i] = inputtrk.par[i];
  for (int i = 0; i < 21; ++i) cov21[i] = inputtrk.cov[i];
  *q = inputtrk.q;
  for (int l = 0; l < 22; ++l) {
    for (int i = 0; i < 3; ++i) hits22x9[l * 9 + i] = inputhits[l].pos[i];
    for (int i = 0; i < 6; ++i) hits22x9[l * 9 + 3 + i] = inputhits[l].cov[i];
  }
}

// Runs the reference program's unmodified main (fixture sizes are this build's macros).
int ref_main(void) { return p2r_tbb_ref_main(0, nullptr); }

}  // extern "C"
