// C-ABI plumbing: error reporting, configuration checks, kfact, and the reference's
// end-of-run validation summary.
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "p2r_internal.h"

namespace {
thread_local char g_last_error[512] = "";
}

int p2r_set_error(int code, const char* msg) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg ? msg : "");
  return code;
}

int p2r_set_errorf(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int p2r_clear_error() {
  g_last_error[0] = '\0';
  return P2R_OK;
}

float p2r_kfact_of(double bz) {
  if (bz == 0.0) bz = 3.8112;  // the reference's compiled-in field (TBB:654)
  return (float)(100 / (-0.299792458 * bz));
}

int p2r_check_aligned(const char* who, unsigned align, std::initializer_list<const void*> ptrs) {
  int i = 0;
  for (const void* p : ptrs) {
    if (p && ((uintptr_t)p % align) != 0)
      return p2r_set_errorf(P2R_ERR_INVALID, "%s: array argument %d is not %u-byte aligned", who, i, align);
    ++i;
  }
  return P2R_OK;
}

int p2r_check_disjoint(const char* who, const char* what, const void* a, size_t na, const void* b, size_t nb,
                       bool allow_same) {
  if (!a || !b || na == 0 || nb == 0) return P2R_OK;
  if (allow_same && a == b && na == nb) return P2R_OK;
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  if (x < y + nb && y < x + na) return p2r_set_errorf(P2R_ERR_INVALID, "%s: %s overlap", who, what);
  return P2R_OK;
}

int p2r_check_spans(const char* who, std::initializer_list<P2rSpan> spans) {
  const P2rSpan* v = spans.begin();
  const size_t n = spans.size();
  for (size_t i = 0; i < n; ++i)
    for (size_t j = i + 1; j < n; ++j) {
      if (!v[i].written && !v[j].written) continue;
      if (!v[i].ptr || !v[j].ptr || v[i].bytes == 0 || v[j].bytes == 0) continue;
      const uintptr_t a = (uintptr_t)v[i].ptr, b = (uintptr_t)v[j].ptr;
      if (a < b + v[j].bytes && b < a + v[i].bytes)
        return p2r_set_errorf(P2R_ERR_INVALID, "%s: %s and %s overlap", who, v[i].name, v[j].name);
    }
  return P2R_OK;
}

int p2r_check_config(const p2r_config* cfg, const char* who) {
  if (!cfg) return p2r_set_errorf(P2R_ERR_INVALID, "%s: config is null", who);
  if (cfg->bsize < 1 || cfg->bsize > 4096)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: bsize %d outside [1, 4096]", who, cfg->bsize);
  if (cfg->nlayer < 1 || cfg->nlayer > 4096)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: nlayer %d outside [1, 4096]", who, cfg->nlayer);
  if (cfg->nevts < 0 || cfg->nb < 0)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: negative nevts/nb", who);
  if (cfg->nb > 0 && cfg->nevts > (int64_t)(INT64_C(1) << 40) / cfg->nb)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: nevts*nb too large", who);
  // one thread per track, at least 32 threads per CTA: the grid stays below 2^31 - 1
  const long long ntr = (long long)cfg->nevts * cfg->nb * cfg->bsize;
  if (ntr > (long long)0x7fffffff * 32)
    return p2r_set_errorf(P2R_ERR_INVALID, "%s: %lld tracks exceed the launch grid", who, ntr);
  if (!std::isfinite(cfg->bz)) return p2r_set_errorf(P2R_ERR_INVALID, "%s: bz is not finite", who);
  return P2R_OK;
}

extern "C" {

int p2r_abi_version(void) { return P2R_ABI_VERSION; }

const char* p2r_last_error_string(void) { return g_last_error; }

float p2r_kfact(double bz) { return p2r_kfact_of(bz); }

// TBB:935-1048: means over finite, non-failed tracks divided by the TOTAL track count,
// failure = more than 100 % relative deviation from the last layer's hit in x, y or z.
int p2r_summary(const void* host_trk, int32_t bsize, int64_t nevts, int64_t nb, const float* host_hit_xyz,
                p2r_summary_stats* out) {
  if (!host_trk || !host_hit_xyz || !out) return p2r_set_error(P2R_ERR_INVALID, "p2r_summary: null pointer");
  if (bsize < 1 || nevts < 0 || nb < 0) return p2r_set_error(P2R_ERR_INVALID, "p2r_summary: bad sizes");
  std::memset(out, 0, sizeof(*out));
  const float* trk = (const float*)host_trk;
  const double hx = host_hit_xyz[0], hy = host_hit_xyz[1], hz = host_hit_xyz[2];
  const double hr = std::sqrt(hx * hx + hy * hy);
  const double n = (double)nevts * nb * bsize;
  if (n == 0) return p2r_clear_error();
  auto get = [&](int64_t b, int it, int ip) { return (double)trk[b * 28 * (int64_t)bsize + ip * bsize + it]; };
  const int64_t nblocks = nevts * nb;
  for (int pass = 0; pass < 2; ++pass) {
    for (int64_t b = 0; b < nblocks; ++b)
      for (int it = 0; it < bsize; ++it) {
        const double x = get(b, it, 0), y = get(b, it, 1), z = get(b, it, 2);
        const double r = std::sqrt(x * x + y * y);
        const double pt = std::fabs(1. / get(b, it, 3)), phi = get(b, it, 4), th = get(b, it, 5);
        const bool finite = std::isfinite(x) && std::isfinite(y) && std::isfinite(z) &&
                            (pass == 1 || (std::isfinite(pt) && std::isfinite(phi) && std::isfinite(th)));
        if (!finite) {
          if (pass == 0) out->nnans++;
          continue;
        }
        if (std::fabs((x - hx) / hx) > 1. || std::fabs((y - hy) / hy) > 1. || std::fabs((z - hz) / hz) > 1.) {
          if (pass == 0) out->nfail++;
          continue;
        }
        if (pass == 0) {
          out->avg_pt += pt;
          out->avg_phi += phi;
          out->avg_theta += th;
          out->avg_x += x;
          out->avg_y += y;
          out->avg_z += z;
          out->avg_r += r;
          out->avg_dx += (x - hx) / x;
          out->avg_dy += (y - hy) / y;
          out->avg_dz += (z - hz) / z;
          out->avg_dr += (r - hr) / r;
        } else {
          out->std_x += (x - out->avg_x) * (x - out->avg_x);
          out->std_y += (y - out->avg_y) * (y - out->avg_y);
          out->std_z += (z - out->avg_z) * (z - out->avg_z);
          out->std_r += (r - out->avg_r) * (r - out->avg_r);
          out->std_dx += ((x - hx) / x - out->avg_dx) * ((x - hx) / x - out->avg_dx);
          out->std_dy += ((y - hy) / y - out->avg_dy) * ((y - hy) / y - out->avg_dy);
          out->std_dz += ((z - hz) / z - out->avg_dz) * ((z - hz) / z - out->avg_dz);
          out->std_dr += ((r - hr) / r - out->avg_dr) * ((r - hr) / r - out->avg_dr);
        }
      }
    if (pass == 0) {
      out->avg_pt /= n;
      out->avg_phi /= n;
      out->avg_theta /= n;
      out->avg_x /= n;
      out->avg_y /= n;
      out->avg_z /= n;
      out->avg_r /= n;
      out->avg_dx /= n;
      out->avg_dy /= n;
      out->avg_dz /= n;
      out->avg_dr /= n;
    }
  }
  out->std_x = std::sqrt(out->std_x / n);
  out->std_y = std::sqrt(out->std_y / n);
  out->std_z = std::sqrt(out->std_z / n);
  out->std_r = std::sqrt(out->std_r / n);
  out->std_dx = std::sqrt(out->std_dx / n);
  out->std_dy = std::sqrt(out->std_dy / n);
  out->std_dz = std::sqrt(out->std_dz / n);
  out->std_dr = std::sqrt(out->std_dr / n);
  return p2r_clear_error();
}

}  // extern "C"
