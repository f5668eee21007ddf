// gdf_io.cpp -- the reference's output files and a binary checkpoint, on
// host arrays in the reference layout (no device work here except through
// the public handle calls of the checkpoint).
//
//   gdf_save_solution  save_solution.f90: Q1.txt .. Q8.txt
//   gdf_save_frame     RK3.f90:29-53, 154-172: one frame appended to
//                      Q1flash.txt .. Q8flash.txt and T.txt
//   gdf_save_xy        save_XY.f90: Xc.txt, Yc.txt, lambda.txt, weight.txt
//   gdf_checkpoint_*   uh, Bx, By, t, dt and the sticky troubled-cell flags
//                      of a handle, with its configuration, in one file
//
// The text files hold one value per line in the reference's loop order
// (mode, then j, then i). Values are written with 17 significant digits
// ("%25.16E"), which reads back to the same double; gfortran's
// list-directed layout differs only in spacing and exponent style, which
// the reference's MATLAB readers (MHD_GDF_plot/*.m, load()) ignore.

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gdf.h"

namespace gdf {
int set_last_error(int code, const char* msg);   // gdf_kernels.cu
}

namespace {

constexpr int NG = 5, NP = 10, NE = 8;
const double kLam[NG] = {-0.9061798459386639927976269, -0.5384693101056830910363144, 0,
                         0.5384693101056830910363144, 0.9061798459386639927976269};
const double kW[NG] = {0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
                       0.4786286704993664680412915, 0.2369268850561890875142640};

std::string join(const char* dir, const char* name) {
  std::string p = dir && *dir ? dir : ".";
  if (p.back() != '/') p += '/';
  return p + name;
}

// uh(i, j, d, n) values of interior cells, d-j-i order, to f
bool write_var(FILE* f, const GdfConfig& c, const double* uh, int n) {
  const size_t NX2 = (size_t)c.nx + 2, NY2 = (size_t)c.ny + 2;
  char buf[64];
  for (int d = 0; d < NP; ++d)
    for (int j = 1; j <= c.ny; ++j)
      for (int i = 1; i <= c.nx; ++i) {
        const int len = std::snprintf(buf, sizeof(buf), "%25.16E\n", uh[i + NX2 * (j + NY2 * (d + 10 * (size_t)n))]);
        if (std::fwrite(buf, 1, (size_t)len, f) != (size_t)len) return false;
      }
  return true;
}

int write_set(const GdfConfig* cfg, const double* uh, const char* dir, const char* suffix, const char* mode) {
  for (int n = 0; n < NE; ++n) {
    const std::string name = "Q" + std::to_string(n + 1) + suffix + ".txt";
    FILE* f = std::fopen(join(dir, name.c_str()).c_str(), mode);
    if (!f) return GDF_ERR_ARG;
    const bool ok = write_var(f, *cfg, uh, n);
    if (std::fclose(f) != 0 || !ok) return GDF_ERR_ARG;
  }
  return GDF_OK;
}

struct CkptHeader {
  char magic[8];
  uint32_t abi, cfg_bytes;
  double t, dt;
};

}  // namespace

extern "C" {

int gdf_save_solution(const GdfConfig* cfg, const double* uh, const char* dir) {
  if (!cfg || !uh || cfg->nx < 1 || cfg->ny < 1) return GDF_ERR_ARG;
  return write_set(cfg, uh, dir, "", "w");
}

int gdf_save_frame(const GdfConfig* cfg, const double* uh, double t, const char* dir, int32_t reset) {
  if (!cfg || !uh || cfg->nx < 1 || cfg->ny < 1) return GDF_ERR_ARG;
  const char* mode = reset ? "w" : "a";
  int rc = write_set(cfg, uh, dir, "flash", mode);
  if (rc) return rc;
  FILE* f = std::fopen(join(dir, "T.txt").c_str(), mode);
  if (!f) return GDF_ERR_ARG;
  const bool ok = std::fprintf(f, "%25.16E\n", t) > 0;
  if (std::fclose(f) != 0 || !ok) return GDF_ERR_ARG;
  return GDF_OK;
}

int gdf_save_xy(const GdfConfig* cfg, const char* dir) {
  if (!cfg || cfg->nx < 1 || cfg->ny < 1) return GDF_ERR_ARG;
  const double hx = (cfg->xb - cfg->xa) / cfg->nx, hy = (cfg->yb - cfg->ya) / cfg->ny;
  const double hx1 = 0.5 * hx, hy1 = 0.5 * hy;
  const char* names[4] = {"Xc.txt", "Yc.txt", "lambda.txt", "weight.txt"};
  for (int k = 0; k < 4; ++k) {
    FILE* f = std::fopen(join(dir, names[k]).c_str(), "w");
    if (!f) return GDF_ERR_ARG;
    bool ok = true;
    if (k == 0)
      for (int i = 1; i <= cfg->nx; ++i)
        for (int a = 0; a < NG; ++a) ok = ok && std::fprintf(f, "%25.16E\n", (cfg->xa + (i - 0.5) * hx) + hx1 * kLam[a]) > 0;
    else if (k == 1)
      for (int j = 1; j <= cfg->ny; ++j)
        for (int b = 0; b < NG; ++b) ok = ok && std::fprintf(f, "%25.16E\n", (cfg->ya + (j - 0.5) * hy) + hy1 * kLam[b]) > 0;
    else
      for (int a = 0; a < NG; ++a) ok = ok && std::fprintf(f, "%25.16E\n", k == 2 ? kLam[a] : kW[a]) > 0;
    if (std::fclose(f) != 0 || !ok) return GDF_ERR_ARG;
  }
  return GDF_OK;
}

int gdf_checkpoint_save(GdfHandle* h, const char* path) {
  if (!h || !path) return GDF_ERR_ARG;
  GdfConfig c;
  int rc = gdf_config_of(h, &c);
  if (rc) return rc;
  const size_t plane = (size_t)(c.nx + 2) * (c.ny + 2);
  std::vector<double> uh(plane * NP * NE), bx((size_t)(c.nx + 1) * c.ny * 3), by((size_t)c.nx * (c.ny + 1) * 3);
  std::vector<int32_t> tr((size_t)c.nx * c.ny);
  CkptHeader hd;
  std::memcpy(hd.magic, "GDFCKPT1", 8);
  hd.abi = GDF_ABI_VERSION;
  hd.cfg_bytes = (uint32_t)sizeof(GdfConfig);
  if ((rc = gdf_download(h, uh.data(), bx.data(), by.data()))) return rc;
  if ((rc = gdf_get_time(h, &hd.t, &hd.dt))) return rc;
  if ((rc = gdf_get_trouble(h, tr.data()))) return rc;
  FILE* f = std::fopen(path, "wb");
  if (!f) return gdf::set_last_error(GDF_ERR_ARG, "cannot open the checkpoint file for writing");
  bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 && std::fwrite(&c, sizeof(c), 1, f) == 1 &&
            std::fwrite(uh.data(), sizeof(double), uh.size(), f) == uh.size() &&
            std::fwrite(bx.data(), sizeof(double), bx.size(), f) == bx.size() &&
            std::fwrite(by.data(), sizeof(double), by.size(), f) == by.size() &&
            std::fwrite(tr.data(), sizeof(int32_t), tr.size(), f) == tr.size();
  if (std::fclose(f) != 0) ok = false;
  return ok ? GDF_OK : gdf::set_last_error(GDF_ERR_ARG, "writing the checkpoint failed");
}

int gdf_checkpoint_load(GdfHandle* h, const char* path) {
  if (!h || !path) return GDF_ERR_ARG;
  GdfConfig c, cf;
  int rc = gdf_config_of(h, &c);
  if (rc) return rc;
  FILE* f = std::fopen(path, "rb");
  if (!f) return gdf::set_last_error(GDF_ERR_ARG, "cannot open the checkpoint file");
  CkptHeader hd;
  bool ok = std::fread(&hd, sizeof(hd), 1, f) == 1 && std::memcmp(hd.magic, "GDFCKPT1", 8) == 0 &&
            hd.abi == GDF_ABI_VERSION && hd.cfg_bytes == sizeof(GdfConfig) && std::fread(&cf, sizeof(cf), 1, f) == 1 &&
            std::memcmp(&cf, &c, sizeof(GdfConfig)) == 0;
  const size_t plane = (size_t)(c.nx + 2) * (c.ny + 2);
  std::vector<double> uh(plane * NP * NE), bx((size_t)(c.nx + 1) * c.ny * 3), by((size_t)c.nx * (c.ny + 1) * 3);
  std::vector<int32_t> tr((size_t)c.nx * c.ny);
  ok = ok && std::fread(uh.data(), sizeof(double), uh.size(), f) == uh.size() &&
       std::fread(bx.data(), sizeof(double), bx.size(), f) == bx.size() &&
       std::fread(by.data(), sizeof(double), by.size(), f) == by.size() &&
       std::fread(tr.data(), sizeof(int32_t), tr.size(), f) == tr.size();
  std::fclose(f);
  if (!ok)
    return gdf::set_last_error(GDF_ERR_ARG, "not a checkpoint of this handle's configuration, or a truncated file");
  if ((rc = gdf_upload(h, uh.data(), bx.data(), by.data()))) return rc;
  if ((rc = gdf_set_trouble(h, tr.data()))) return rc;
  return gdf_set_time(h, hd.t);
}

}  // extern "C"
