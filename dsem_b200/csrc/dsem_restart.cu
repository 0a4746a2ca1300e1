// dsem_restart.cu -- DSEM restart files read and written from the device state:
// write_restart / read_restart (src/Parabolic3D/stac3m/restart.f90:19-312,
// 319-929), the branch without `defined_resolution`.
//
// The file is Fortran unformatted sequential: every WRITE statement is one
// record, framed by its length in bytes as a 4-byte little-endian integer
// before and after it.  The record sequence:
//   header       (ngrid, nmort - nmortd), then 12 records of operator
//                matrices and their maps (restart.f90:63-78)
//   per element  24 records (restart.f90:110-137): type, node, orientation,
//                mortar, which_surface, (nc, ncg), Q, Qlgg, Qglg, Qggl, f, g,
//                h, g_Q, material_id, (cx, cxg), xg, jacob, gmet, gmetg,
//                corner, ibtype, bcond, domain_type
//   per mortar   13 records (restart.f90:167-179)
//   then         num_prop and max_materials property records (:187-191), the
//                case's write_restart_case (for the Taylor-Green case one
//                record, the time: caseFiles/tgv/BackstepProblem-stoch.f90:
//                1876-1895), statistics and particles when enabled.
// Q, Qlgg, Qglg, Qggl and g_Q are DIMENSION(nx,ny,nz,neq), neq = 5, with
// nx = ny = nz (size.f90); the element's Gauss counts are its ncg.
//
// dsem_write_restart copies a restart file DSEM wrote for the same mesh (the
// serial zero-step run of DSEM's restart workflow, mainpage.f90:109-125, or
// an earlier restart) record by record, replacing each element's Q, g_Q and,
// when the context keeps them, its three Lobatto arrays by the device state;
// all other records (geometry, mortars, materials, statistics) pass through
// unchanged, and the case record takes the given time.  dsem_read_restart
// uploads Q and, when the file's Lobatto arrays were computed, rebuilds the
// gradients the next step's entropy viscosity and Smagorinsky model use.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dsem_gpu.h"
#include "dsem_ctx.h"

namespace {

constexpr int HEADER_RECORDS = 13;    // (ngrid, nmort) + 12 matrix records
constexpr int ELEMENT_RECORDS = 24;   // restart.f90:110-137
constexpr int MORTAR_RECORDS = 13;    // restart.f90:167-179
constexpr int R_NCG = 5, R_Q = 6, R_QLGG = 7, R_GQ = 13;  // 0-based record indices within an element

struct File {
  FILE *f = nullptr;
  explicit File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

// one record: returns false at a clean end of file, sets err on a malformed record
bool read_record(FILE *f, std::vector<char> &buf, std::string &err) {
  int32_t n = 0, m = 0;
  if (std::fread(&n, 4, 1, f) != 1) return false;
  if (n < 0) {
    err = "record longer than 2 GiB (split records are not supported)";
    return false;
  }
  buf.resize((size_t)n);
  if ((n > 0 && std::fread(buf.data(), 1, (size_t)n, f) != (size_t)n) || std::fread(&m, 4, 1, f) != 1 || m != n) {
    err = "truncated or malformed record";
    return false;
  }
  return true;
}

bool write_record(FILE *f, const char *data, size_t n) {
  const int32_t m = (int32_t)n;
  return std::fwrite(&m, 4, 1, f) == 1 && (n == 0 || std::fwrite(data, 1, n, f) == n) && std::fwrite(&m, 4, 1, f) == 1;
}

// nx of a (nx,nx,nx,5) double record
int padded_nx(size_t bytes) {
  if (bytes % 40) return -1;
  const long long n3 = (long long)(bytes / 40);
  long long nx = (long long)std::llround(std::cbrt((double)n3));
  return nx * nx * nx == n3 ? (int)nx : -1;
}

// grid d of element order G (L = G+1 points along d) <-> DSEM (nx,nx,nx,5) record
template <bool TO_RECORD>
void lob_copy(double *rec, int nx, double *lob, int G, int d) {
  const int L = G + 1, ex = d == 0 ? L : G, ey = d == 1 ? L : G, ez = d == 2 ? L : G;
  const size_t nl = (size_t)L * G * G, n3 = (size_t)nx * nx * nx;
  for (int v = 0; v < 5; ++v)
    for (int z = 0; z < ez; ++z)
      for (int y = 0; y < ey; ++y)
        for (int x = 0; x < ex; ++x) {
          double &r = rec[v * n3 + x + (size_t)nx * (y + (size_t)nx * z)];
          double &l = lob[v * nl + x + (size_t)ex * (y + (size_t)ey * z)];
          if (TO_RECORD)
            r = l;
          else
            l = r;
        }
}

int rfail(dsem_ctx *c, int code, const std::string &msg) { return dsem_int::fail(c, code, "restart file: " + msg); }

int check_ctx(dsem_ctx *c) {
  if (!c) return DSEM_ERR_INVALID_ARG;
  if (c->ncase != 1) return rfail(c, DSEM_ERR_UNSUPPORTED, "one case per context (ensembles are not supported)");
  if (c->ncut) return rfail(c, DSEM_ERR_UNSUPPORTED, "sharded contexts are not supported");
  return DSEM_OK;
}

// element e's Gauss counts from its (nc, ncg) record
bool ncg_matches(const std::vector<char> &b, int G) {
  if (b.size() != 24) return false;
  int32_t v[6];
  std::memcpy(v, b.data(), 24);
  return v[3] == G && v[4] == G && v[5] == G;
}

}  // namespace

extern "C" {

int dsem_write_restart(dsem_ctx *c, const char *template_path, const char *out_path, int max_materials,
                       double time) {
  int r = check_ctx(c);
  if (r) return r;
  if (!template_path || !out_path) return rfail(c, DSEM_ERR_INVALID_ARG, "null path");
  if (max_materials < 0) return rfail(c, DSEM_ERR_INVALID_ARG, "max_materials < 0");
  File in(template_path, "rb");
  if (!in.f) return rfail(c, DSEM_ERR_INVALID_ARG, std::string("cannot open template ") + template_path);
  std::vector<char> rec;
  std::string err;
  // header
  std::vector<std::vector<char>> head;
  for (int i = 0; i < HEADER_RECORDS; ++i) {
    if (!read_record(in.f, rec, err)) return rfail(c, DSEM_ERR_INVALID_ARG, err.empty() ? "header truncated" : err);
    head.push_back(rec);
  }
  int32_t hdr[2];
  if (head[0].size() != 8) return rfail(c, DSEM_ERR_INVALID_ARG, "first record is not (ngrid, nmort)");
  std::memcpy(hdr, head[0].data(), 8);
  if (hdr[0] != c->ngrid) return rfail(c, DSEM_ERR_INVALID_ARG, "template has another element count");
  // device state in the caller's layout (nx from the template's Q record, known after element 1)
  std::vector<double> q, gq, lob;
  std::vector<long long> loff;
  const bool with_lob = c->keep_lob && c->lob_valid;
  if (with_lob) {
    loff = dsem_int::lob_offsets(c);
    lob.resize((size_t)loff.back());
    if ((r = dsem_int::lob_download(c, lob.data()))) return r;
  }
  File out(out_path, "wb");
  if (!out.f) return rfail(c, DSEM_ERR_INVALID_ARG, std::string("cannot create ") + out_path);
  for (auto &h : head)
    if (!write_record(out.f, h.data(), h.size())) return rfail(c, DSEM_ERR_INVALID_ARG, "write failed");
  int nx = -1;
  for (int e = 0; e < c->ngrid; ++e) {
    const int G = c->groups[c->ext_group[e]].G;
    for (int k = 0; k < ELEMENT_RECORDS; ++k) {
      if (!read_record(in.f, rec, err)) return rfail(c, DSEM_ERR_INVALID_ARG, err.empty() ? "element records truncated" : err);
      if (k == R_NCG && !ncg_matches(rec, G)) return rfail(c, DSEM_ERR_INVALID_ARG, "element order differs from the template's ncg");
      if (k >= R_Q && k <= R_GQ) {
        const int n = padded_nx(rec.size());
        if (k == R_Q) {
          if (n < G) return rfail(c, DSEM_ERR_INVALID_ARG, "Q record is not (nx,nx,nx,5) with nx >= p+1");
          if (nx < 0) {
            nx = n;
            const size_t L3 = (size_t)nx * nx * nx;
            q.resize((size_t)c->ngrid * 5 * L3);
            gq.resize(q.size());
            if ((r = dsem_download_q(c, q.data(), nx))) return r;
            if ((r = dsem_int::unpack_state(c, c->gQ, gq.data(), nx))) return r;
          } else if (n != nx) {
            return rfail(c, DSEM_ERR_INVALID_ARG, "Q records of different sizes");
          }
        }
        const size_t L3 = (size_t)nx * nx * nx;
        if (k == R_Q) {
          std::vector<double> tmp(rec.size() / 8);
          std::memcpy(tmp.data(), rec.data(), rec.size());
          for (int v = 0; v < 5; ++v)  // the Gauss points; the padding keeps the template's values
            for (int z = 0; z < G; ++z)
              for (int y = 0; y < G; ++y)
                for (int x = 0; x < G; ++x) {
                  const size_t i = v * L3 + x + (size_t)nx * (y + (size_t)nx * z);
                  tmp[i] = q[(size_t)e * 5 * L3 + i];
                }
          std::memcpy(rec.data(), tmp.data(), rec.size());
        } else if (k == R_GQ && padded_nx(rec.size()) == nx) {
          std::vector<double> tmp(rec.size() / 8);
          std::memcpy(tmp.data(), rec.data(), rec.size());
          for (int v = 0; v < 5; ++v)
            for (int z = 0; z < G; ++z)
              for (int y = 0; y < G; ++y)
                for (int x = 0; x < G; ++x) {
                  const size_t i = v * L3 + x + (size_t)nx * (y + (size_t)nx * z);
                  tmp[i] = gq[(size_t)e * 5 * L3 + i];
                }
          std::memcpy(rec.data(), tmp.data(), rec.size());
        } else if (with_lob && k >= R_QLGG && k < R_QLGG + 3) {
          if (padded_nx(rec.size()) != nx || nx < G + 1)
            return rfail(c, DSEM_ERR_INVALID_ARG, "Lobatto record is not (nx,nx,nx,5) with nx >= p+2");
          std::vector<double> tmp(rec.size() / 8);
          std::memcpy(tmp.data(), rec.data(), rec.size());
          const int d = k - R_QLGG;
          lob_copy<true>(tmp.data(), nx, lob.data() + loff[e] + (size_t)d * 5 * (G + 1) * G * G, G, d);
          std::memcpy(rec.data(), tmp.data(), rec.size());
        }
      }
      if (!write_record(out.f, rec.data(), rec.size())) return rfail(c, DSEM_ERR_INVALID_ARG, "write failed");
    }
  }
  // mortars, material properties: through; the case record takes the time
  const int32_t nm = hdr[1];
  for (int i = 0; i < nm * MORTAR_RECORDS; ++i) {
    if (!read_record(in.f, rec, err)) return rfail(c, DSEM_ERR_INVALID_ARG, err.empty() ? "mortar records truncated" : err);
    if (!write_record(out.f, rec.data(), rec.size())) return rfail(c, DSEM_ERR_INVALID_ARG, "write failed");
  }
  if (!read_record(in.f, rec, err) || rec.size() != 4) return rfail(c, DSEM_ERR_INVALID_ARG, "num_prop record missing");
  if (!write_record(out.f, rec.data(), rec.size())) return rfail(c, DSEM_ERR_INVALID_ARG, "write failed");
  // max_materials property records (size.f90), then the case's records: the first is the
  // time for DSEM's Taylor-Green and isotropic cases; statistics and particles follow
  for (int i = 0; i < max_materials; ++i) {
    if (!read_record(in.f, rec, err)) return rfail(c, DSEM_ERR_INVALID_ARG, err.empty() ? "property records truncated" : err);
    if (!write_record(out.f, rec.data(), rec.size())) return rfail(c, DSEM_ERR_INVALID_ARG, "write failed");
  }
  bool first = true;
  while (read_record(in.f, rec, err)) {
    if (first && rec.size() == 8) std::memcpy(rec.data(), &time, 8);
    first = false;
    if (!write_record(out.f, rec.data(), rec.size())) return rfail(c, DSEM_ERR_INVALID_ARG, "write failed");
  }
  if (!err.empty()) return rfail(c, DSEM_ERR_INVALID_ARG, err);
  if (std::fflush(out.f) != 0) return rfail(c, DSEM_ERR_INVALID_ARG, "write failed");
  return DSEM_OK;
}

int dsem_read_restart(dsem_ctx *c, const char *path, int max_materials, double *time) {
  int r = check_ctx(c);
  if (r) return r;
  if (!path) return rfail(c, DSEM_ERR_INVALID_ARG, "null path");
  if (max_materials < 0) return rfail(c, DSEM_ERR_INVALID_ARG, "max_materials < 0");
  File in(path, "rb");
  if (!in.f) return rfail(c, DSEM_ERR_INVALID_ARG, std::string("cannot open ") + path);
  std::vector<char> rec;
  std::string err;
  if (!read_record(in.f, rec, err) || rec.size() != 8) return rfail(c, DSEM_ERR_INVALID_ARG, "first record is not (ngrid, nmort)");
  int32_t hdr[2];
  std::memcpy(hdr, rec.data(), 8);
  if (hdr[0] != c->ngrid) return rfail(c, DSEM_ERR_INVALID_ARG, "file has another element count");
  for (int i = 1; i < HEADER_RECORDS; ++i)
    if (!read_record(in.f, rec, err)) return rfail(c, DSEM_ERR_INVALID_ARG, err.empty() ? "header truncated" : err);
  const auto loff = dsem_int::lob_offsets(c);
  std::vector<double> q, lob((size_t)loff.back(), 0.0);
  bool any_lob = false;
  int nx = -1;
  for (int e = 0; e < c->ngrid; ++e) {
    const int G = c->groups[c->ext_group[e]].G;
    for (int k = 0; k < ELEMENT_RECORDS; ++k) {
      if (!read_record(in.f, rec, err)) return rfail(c, DSEM_ERR_INVALID_ARG, err.empty() ? "element records truncated" : err);
      if (k == R_NCG && !ncg_matches(rec, G)) return rfail(c, DSEM_ERR_INVALID_ARG, "element order differs from the file's ncg");
      if (k == R_Q) {
        const int n = padded_nx(rec.size());
        if (n < G || (nx >= 0 && n != nx)) return rfail(c, DSEM_ERR_INVALID_ARG, "Q record is not (nx,nx,nx,5)");
        if (nx < 0) {
          nx = n;
          q.resize((size_t)c->ngrid * 5 * nx * nx * nx);
        }
        std::memcpy(q.data() + (size_t)e * 5 * nx * nx * nx, rec.data(), rec.size());
      } else if (k >= R_QLGG && k < R_QLGG + 3) {
        if (padded_nx(rec.size()) != nx || nx < G + 1)
          return rfail(c, DSEM_ERR_INVALID_ARG, "Lobatto record is not (nx,nx,nx,5) with nx >= p+2");
        std::vector<double> tmp(rec.size() / 8);
        std::memcpy(tmp.data(), rec.data(), rec.size());
        const int d = k - R_QLGG;
        double *l = lob.data() + loff[e] + (size_t)d * 5 * (G + 1) * G * G;
        lob_copy<false>(tmp.data(), nx, l, G, d);
        for (size_t i = 0; i < (size_t)5 * (G + 1) * G * G && !any_lob; ++i) any_lob = l[i] != 0.0;
      }
    }
  }
  const int32_t nm = hdr[1];
  for (int i = 0; i < nm * MORTAR_RECORDS; ++i)
    if (!read_record(in.f, rec, err)) return rfail(c, DSEM_ERR_INVALID_ARG, err.empty() ? "mortar records truncated" : err);
  if (!read_record(in.f, rec, err) || rec.size() != 4) return rfail(c, DSEM_ERR_INVALID_ARG, "num_prop record missing");
  for (int i = 0; i < max_materials; ++i)
    if (!read_record(in.f, rec, err)) return rfail(c, DSEM_ERR_INVALID_ARG, err.empty() ? "property records truncated" : err);
  double t = 0.0;
  if (read_record(in.f, rec, err) && rec.size() == 8) std::memcpy(&t, rec.data(), 8);
  if (time) *time = t;
  if ((r = dsem_upload_q(c, q.data(), nx))) return r;
  // DSEM's zero-step file holds zeroed Lobatto arrays (zero_domain): no valid gradients, so
  // the first step's entropy viscosity is 0, as on a fresh start
  if (any_lob) return dsem_int::lob_upload_grad(c, lob.data());
  dsem_int::grad_invalidate(c);
  return DSEM_OK;
}

}  // extern "C"
