// lce_confio.cu -- configurations in the reference's direct-access format,
// and the reference's output file names.
//
// f/confsave.f:57-233 / f/confget.f:349-526 write and read one unformatted
// direct-access record per (mu, eo, z) for the links and per (eo, z) for the
// Higgs field.  A record holds one global xy slice of one parity in half-row
// order (x fastest): L1*L2/2 sites of COMPLEX(2) (links) or REAL(3) (A0), in
// single precision.  The record lengths the reference declares,
//   u_rl = 16 * nc * L1*L2/2 bytes,   a_rl = 8 * 3 * L1*L2/2 bytes,
// are twice the payload; the rest of each record is zero here.
//
// Resume: the reference names saved files with "_BE".."_U" (f/confsave.f:249-253)
// but reads "_be".."_u" (f/measinit.f:246-250), and it never restores its
// random-number state.  Here both directions use the lower-case names and a
// sidecar "<u file>.rng" records the Philox pass counter (and the validation
// stream position), so a resumed run with the same seed continues the same
// random stream.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lce_internal.hpp"

extern "C" int lce_conf_filename(char* buf, size_t n, const char* prefix, int L3, double beta, double x, double y,
                                 int number) {
  if (!buf || !prefix || n == 0) return LCE_ERR_INVALID;
  // f/measinit.f:240 format: '<prefix>_s', i2.2, '_be', i5.5, '_x', i5.5, '_y', i5.5, '_u', i6.6
  const long betaint = std::lround(1000.0 * beta), xint = std::lround(10000.0 * x), yint = std::lround(10000.0 * y);
  const int r = std::snprintf(buf, n, "%s_s%02d_be%05ld_x%05ld_y%05ld_u%06d", prefix, L3, betaint, xint, yint, number);
  return (r < 0 || (size_t)r >= n) ? LCE_ERR_INVALID : LCE_OK;
}

extern "C" int lce_confsave(lce_ctx* c, int chain, const char* u_path, const char* a_path) {
  if (!c || !u_path || !a_path) return LCE_ERR_INVALID;
  int L[3];
  int rc0 = lce_get_extents(c, chain, L);
  if (rc0) return rc0;
  const int L1 = L[0], L2 = L[1], L3 = L[2];
  const long nxy = (long)L1 * L2 / 2, nh = nxy * L3;
  std::vector<float> u((size_t)24 * nh), a((size_t)6 * nh);
  int rc = lce_download(c, chain, LCE_FIELDS, u.data(), a.data(), nh);
  if (rc) return rc;
  FILE* fu = std::fopen(u_path, "wb");
  FILE* fa = fu ? std::fopen(a_path, "wb") : nullptr;
  if (!fu || !fa) {
    if (fu) std::fclose(fu);
    lce::set_thread_error(std::string("lce_confsave: cannot open ") + (fu ? a_path : u_path));
    return LCE_ERR_INVALID;
  }
  bool ok = true;
  // links: records (mu, eo, z); payload nxy * 4 floats, record 2x payload
  std::vector<float> pad((size_t)8 * nxy, 0.0f);
  for (int mu = 0; mu < 3 && ok; ++mu)
    for (int eo = 0; eo < 2 && ok; ++eo)
      for (int z = 0; z < L3 && ok; ++z) {
        const float* src = u.data() + (((size_t)(mu * 2 + eo)) * nh + (size_t)z * nxy) * 4;
        std::memcpy(pad.data(), src, sizeof(float) * 4 * nxy);
        ok = std::fwrite(pad.data(), sizeof(float), pad.size(), fu) == pad.size();
      }
  std::vector<float> apad((size_t)6 * nxy, 0.0f);
  for (int eo = 0; eo < 2 && ok; ++eo)
    for (int z = 0; z < L3 && ok; ++z) {
      const float* src = a.data() + ((size_t)eo * nh + (size_t)z * nxy) * 3;
      std::memcpy(apad.data(), src, sizeof(float) * 3 * nxy);
      ok = std::fwrite(apad.data(), sizeof(float), apad.size(), fa) == apad.size();
    }
  ok = (std::fclose(fu) == 0) && ok;
  ok = (std::fclose(fa) == 0) && ok;
  if (!ok) {
    lce::set_thread_error("lce_confsave: write failed");
    return LCE_ERR_INVALID;
  }
  unsigned long long pass_ctr = 0, stream_pos = 0;
  rc = lce_get_rng_position(c, &pass_ctr, &stream_pos);
  if (rc) return rc;
  FILE* fr = std::fopen((std::string(u_path) + ".rng").c_str(), "w");
  if (!fr) {
    lce::set_thread_error("lce_confsave: cannot write the .rng sidecar");
    return LCE_ERR_INVALID;
  }
  std::fprintf(fr, "philox_pass_counter %llu\nstream_position %llu\n", pass_ctr, stream_pos);
  std::fclose(fr);
  return LCE_OK;
}

extern "C" int lce_confget(lce_ctx* c, int chain, const char* u_path, const char* a_path) {
  if (!c || !u_path || !a_path) return LCE_ERR_INVALID;
  int L[3];
  int rc0 = lce_get_extents(c, chain, L);
  if (rc0) return rc0;
  const int L1 = L[0], L2 = L[1], L3 = L[2];
  const long nxy = (long)L1 * L2 / 2, nh = nxy * L3;
  std::vector<float> u((size_t)24 * nh), a((size_t)6 * nh);
  FILE* fu = std::fopen(u_path, "rb");
  FILE* fa = fu ? std::fopen(a_path, "rb") : nullptr;
  if (!fu || !fa) {
    if (fu) std::fclose(fu);
    lce::set_thread_error(std::string("lce_confget: cannot open ") + (fu ? a_path : u_path));
    return LCE_ERR_INVALID;
  }
  bool ok = true;
  std::vector<float> rec((size_t)8 * nxy);
  for (int mu = 0; mu < 3 && ok; ++mu)
    for (int eo = 0; eo < 2 && ok; ++eo)
      for (int z = 0; z < L3 && ok; ++z) {
        // the payload is the first half of the record; the last record may be short
        const size_t got = std::fread(rec.data(), sizeof(float), rec.size(), fu);
        ok = got >= (size_t)4 * nxy;
        if (ok) std::memcpy(u.data() + (((size_t)(mu * 2 + eo)) * nh + (size_t)z * nxy) * 4, rec.data(),
                            sizeof(float) * 4 * nxy);
      }
  std::vector<float> arec((size_t)6 * nxy);
  for (int eo = 0; eo < 2 && ok; ++eo)
    for (int z = 0; z < L3 && ok; ++z) {
      const size_t got = std::fread(arec.data(), sizeof(float), arec.size(), fa);
      ok = got >= (size_t)3 * nxy;
      if (ok) std::memcpy(a.data() + ((size_t)eo * nh + (size_t)z * nxy) * 3, arec.data(), sizeof(float) * 3 * nxy);
    }
  std::fclose(fu);
  std::fclose(fa);
  if (!ok) {
    lce::set_thread_error("lce_confget: configuration file shorter than the lattice (truncated or wrong size)");
    return LCE_ERR_INVALID;
  }
  for (float v : u)
    if (!std::isfinite(v)) {
      lce::set_thread_error("lce_confget: non-finite link component in the file");
      return LCE_ERR_NAN;
    }
  int rc = lce_upload(c, chain, LCE_FIELDS, u.data(), a.data(), nh);
  if (rc) return rc;
  FILE* fr = std::fopen((std::string(u_path) + ".rng").c_str(), "r");
  if (fr) {
    unsigned long long pc = 0, sp = 0;
    const int n = std::fscanf(fr, "philox_pass_counter %llu stream_position %llu", &pc, &sp);
    std::fclose(fr);
    if (n == 2) return lce_set_rng_position(c, pc, sp);
  }
  return LCE_OK;
}
