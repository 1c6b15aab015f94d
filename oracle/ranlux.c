/*
 * ranlux.c -- restatement of the RANLUX generator of f/luxury.f
 * (Marsaglia-Zaman subtract-with-borrow with Luescher's luxury skipping).
 *
 * TEST INFRASTRUCTURE ONLY (part of the oracle).  The reference uses it to
 * seed gfortran's random_number (f/measinit.f:214-217); the oracle also uses
 * it as a host-side uniform stream for validation mode.
 *
 * Arithmetic is single precision, as in the Fortran (default REAL), so the
 * outputs reproduce the expected values pinned in f/luxtst.f:88-162.
 * State lives in file-scope statics, mirroring the /LUX1/ and /LUX2/ COMMON
 * blocks of f/luxury.h.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include "lce_oracle.h"

enum { MAXLEV = 4, LXDFLT = 3 };
static const int JSDFLT = 314159265;
static const int IGIGA = 1000000000;
static const float TWOP12 = 4096.0f;
static const int ITWO24 = 1 << 24;
static const int ICONS = 2147483563;
static const int NDSKIP[MAXLEV + 1] = {0, 24, 73, 199, 365};

static int notyet = 1;
static int i24 = 24, j24 = 10, luxlev = LXDFLT;
static float carry = 0.0f;
static float seeds[25];          /* 1-based like the Fortran */
static float twom24, twom12;
static int nskip, in24 = 0, next_[25], kount = 0, mkount = 0, inseed;

/* one subtract-with-borrow step, f/luxury.f:69-78 */
static inline float swb_step(void) {
  float uni = seeds[j24] - seeds[i24] - carry;
  if (uni < 0.0f) {
    uni = uni + 1.0f;
    carry = twom24;
  } else {
    carry = 0.0f;
  }
  seeds[i24] = uni;
  i24 = next_[i24];
  j24 = next_[j24];
  return uni;
}

/* 24 LCG-derived seeds, f/luxury.f:44-51 and :246-253 */
static void seed_from_int(int jseed) {
  int iseeds[25];
  twom24 = 1.0f;
  for (int i = 1; i <= 24; ++i) {
    twom24 = twom24 * 0.5f;
    int k = jseed / 53668;
    jseed = 40014 * (jseed - k * 53668) - k * 12211;
    if (jseed < 0) jseed = jseed + ICONS;
    iseeds[i] = jseed % ITWO24;
  }
  twom12 = twom24 * 4096.0f;
  for (int i = 1; i <= 24; ++i) {
    seeds[i] = (float)iseeds[i] * twom24;
    next_[i] = i - 1;
  }
  next_[1] = 24;
  i24 = 24;
  j24 = 10;
  carry = 0.0f;
  if (seeds[24] == 0.0f) carry = twom24;
}

void lco_ranlux_default(void) {
  notyet = 1;
  i24 = 24; j24 = 10; luxlev = LXDFLT;
  in24 = 0; kount = 0; mkount = 0; carry = 0.0f;
}

/* f/luxury.f:12-112 */
void lco_ranlux(float *rvec, int lenv) {
  if (notyet) {
    notyet = 0;
    int jseed = JSDFLT;
    inseed = jseed;
    luxlev = LXDFLT;
    nskip = NDSKIP[luxlev];
    in24 = 0;
    kount = 0;
    mkount = 0;
    seed_from_int(jseed);
  }
  for (int ivec = 0; ivec < lenv; ++ivec) {
    float uni = swb_step();
    rvec[ivec] = uni;
    if (uni < twom12) {
      rvec[ivec] = rvec[ivec] + twom24 * seeds[j24];
      if (rvec[ivec] == 0.0f) rvec[ivec] = twom24 * twom24;
    }
    in24 = in24 + 1;
    if (in24 == 24) {
      in24 = 0;
      kount = kount + nskip;
      for (int isk = 0; isk < nskip; ++isk) (void)swb_step();
    }
  }
  kount = kount + lenv;
  if (kount >= IGIGA) {
    mkount = mkount + 1;
    kount = kount - IGIGA;
  }
}

/* f/luxury.f:116-165 */
void lco_rluxin(const int32_t isdext[25]) {
  notyet = 0;
  twom24 = 1.0f;
  for (int i = 1; i <= 24; ++i) {
    next_[i] = i - 1;
    twom24 = twom24 * 0.5f;
  }
  next_[1] = 24;
  twom12 = twom24 * 4096.0f;
  for (int i = 1; i <= 24; ++i) seeds[i] = (float)isdext[i - 1] * twom24;
  carry = 0.0f;
  if (isdext[24] < 0) carry = twom24;
  int isd = abs(isdext[24]);
  i24 = isd % 100;
  isd = isd / 100;
  j24 = isd % 100;
  isd = isd / 100;
  in24 = isd % 100;
  isd = isd / 100;
  luxlev = isd;
  if (luxlev <= MAXLEV) {
    nskip = NDSKIP[luxlev];
  } else if (luxlev >= 24) {
    nskip = luxlev - 24;
  } else {
    nskip = NDSKIP[MAXLEV];
    luxlev = MAXLEV;
  }
  inseed = -1;
}

/* f/luxury.f:169-183 */
void lco_rluxut(int32_t isdext[25]) {
  for (int i = 1; i <= 24; ++i) isdext[i - 1] = (int32_t)(seeds[i] * TWOP12 * TWOP12);
  isdext[24] = i24 + 100 * j24 + 10000 * in24 + 1000000 * luxlev;
  if (carry > 0.0f) isdext[24] = -isdext[24];
}

/* f/luxury.f:187-197 */
void lco_rluxat(int *lout, int *inout, int *k1, int *k2) {
  *lout = luxlev;
  *inout = inseed;
  *k1 = kount;
  *k2 = mkount;
}

/* f/luxury.f:201-303 */
void lco_rluxgo(int lux, int ins, int k1, int k2) {
  if (lux < 0) {
    luxlev = LXDFLT;
  } else if (lux <= MAXLEV) {
    luxlev = lux;
  } else if (lux < 24 || lux > 2000) {
    luxlev = MAXLEV;
  } else {
    luxlev = lux;
    for (int ilx = 0; ilx <= MAXLEV; ++ilx)
      if (lux == NDSKIP[ilx] + 24) luxlev = ilx;
  }
  if (luxlev <= MAXLEV) nskip = NDSKIP[luxlev];
  else nskip = luxlev - 24;
  in24 = 0;
  int jseed = (ins > 0) ? ins : JSDFLT;
  inseed = jseed;
  notyet = 0;
  seed_from_int(jseed);
  kount = k1;
  mkount = k2;
  if (k1 + k2 != 0) {
    for (int iouter = 1; iouter <= k2 + 1; ++iouter) {
      int inner = IGIGA;
      if (iouter == k2 + 1) inner = k1;
      for (int isk = 0; isk < inner; ++isk) (void)swb_step();
    }
    in24 = kount % (nskip + 24);
    if (mkount > 0) {
      int izip = IGIGA % (nskip + 24);
      int izip2 = mkount * izip + in24;
      in24 = izip2 % (nskip + 24);
    }
    if (in24 > 23) in24 = 0;
  }
}
