// AMReX plotfile output (one level, or the two levels of the AMR driver)
// and input of one level (host code).
//
// A plotfile is a directory holding
//   Header            the plotfile header CAMR::writePlotFile writes
//                     (Source/Utils/CAMR_io.cpp:408-565): type string,
//                     variable names, dimension, time, finest level, problem
//                     box, refinement ratios, domain boxes, level steps, cell
//                     sizes, coordinate system, boundary width, then per level
//                     its grid count, time, step, the physical extent of
//                     every grid and the relative path of its cell data;
//   Level_0/Cell_H    the MultiFab header (VisMF "version 1" layout: how,
//                     component and ghost counts, the box list, the data file
//                     and byte offset of every box, per-box minima and maxima);
//   Level_0/Cell_D_00000
//                     every box as one FAB: an ASCII line naming the real
//                     format (IEEE double, little-endian byte order), the
//                     box and the component count, then the component planes
//                     of the box, i fastest (the Array4 layout).
// Covered cells of an EB level are written as zero (EB_set_covered before
// VisMF::Write, CAMR_io.cpp:556-558): the caller passes the state as it
// holds it, and covered cells already hold zero.
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "camr_b200.h"

namespace {

thread_local std::string g_io_error;

camr_status io_fail(const std::string& why) {
  g_io_error = why;
  return CAMR_ERR_INVALID;
}

bool make_dir(const std::string& d) {
  if (mkdir(d.c_str(), 0755) == 0) return true;
  return errno == EEXIST;
}

std::string box_text(const int lo[3], const int hi[3]) {
  std::ostringstream o;
  o << "((" << lo[0] << ',' << lo[1] << ',' << lo[2] << ") (" << hi[0] << ',' << hi[1] << ','
    << hi[2] << ") (0,0,0))";
  return o.str();
}

// Default names of the state components (Source/Utils/CAMR_setup.cpp:159-198).
const char* const kStateNames[CAMR_NVAR] = {"density", "xmom",  "ymom", "zmom",  "rho_E",
                                            "rho_e",   "Temp",  "rho_F", "rho_A", "rho_P"};

// The FAB real-format line of little-endian IEEE doubles.
const char* const kFabFormat = "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))";

bool host_little_endian() {
  const uint16_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

// One level's grids as the Header describes them.
struct LevelOut {
  int dom_lo[3], dom_hi[3];
  double dx[3];
  int level_step;
  int nbox;
  const int* boxes;  // nbox x (lo0,lo1,lo2,hi0,hi1,hi2)
};

// Level_L/Cell_D_00000 and Level_L/Cell_H of one level.  row(b, c, j, k)
// returns p with p[i] = component c of cell (i, j, k) of box b.
template <class Row>
camr_status write_level_files(const std::string& lev, int nbox, const int* boxes, int ncomp,
                              Row row, const std::string& mf = "Cell") {
  if (!make_dir(lev)) return io_fail("cannot create " + lev);
  const std::string dname = mf + "_D_00000";
  std::vector<int64_t> offs(nbox);
  std::vector<double> mins(size_t(nbox) * ncomp), maxs(size_t(nbox) * ncomp);
  {
    std::FILE* f = std::fopen((lev + "/" + dname).c_str(), "wb");
    if (!f) return io_fail("cannot write " + lev + "/" + dname);
    std::vector<double> buf;
    int64_t pos = 0;
    for (int b = 0; b < nbox; ++b) {
      const int* lo = boxes + 6 * b;
      const int* hi = boxes + 6 * b + 3;
      const int bn[3] = {hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1};
      const int64_t bc = int64_t(bn[0]) * bn[1] * bn[2];
      offs[b] = pos;
      std::ostringstream h;
      h << kFabFormat << box_text(lo, hi) << ' ' << ncomp << '\n';
      const std::string hs = h.str();
      std::fwrite(hs.data(), 1, hs.size(), f);
      pos += int64_t(hs.size());
      buf.resize(size_t(bc));
      for (int c = 0; c < ncomp; ++c) {
        double mn = std::numeric_limits<double>::max();
        double mx = std::numeric_limits<double>::lowest();
        int64_t t = 0;
        for (int k = lo[2]; k <= hi[2]; ++k)
          for (int j = lo[1]; j <= hi[1]; ++j) {
            const double* r = row(b, c, j, k);
            for (int i = lo[0]; i <= hi[0]; ++i) {
              const double v = r[i];
              buf[size_t(t++)] = v;
              mn = v < mn ? v : mn;
              mx = v > mx ? v : mx;
            }
          }
        mins[size_t(b) * ncomp + c] = mn;
        maxs[size_t(b) * ncomp + c] = mx;
        std::fwrite(buf.data(), sizeof(double), size_t(bc), f);
        pos += bc * int64_t(sizeof(double));
      }
    }
    if (std::fclose(f) != 0) return io_fail("write failed: " + lev + "/" + dname);
  }
  std::ofstream h(lev + "/" + mf + "_H");
  if (!h) return io_fail("cannot write " + lev + "/" + mf + "_H");
  h << 1 << '\n' << 1 << '\n' << ncomp << '\n' << 0 << '\n';
  h << '(' << nbox << " 0\n";
  for (int b = 0; b < nbox; ++b) h << box_text(boxes + 6 * b, boxes + 6 * b + 3) << '\n';
  h << ")\n" << nbox << '\n';
  for (int b = 0; b < nbox; ++b) h << "FabOnDisk: " << dname << ' ' << offs[b] << '\n';
  h << '\n' << nbox << ',' << ncomp << '\n';
  h << std::setprecision(17);
  for (int b = 0; b < nbox; ++b) {
    for (int c = 0; c < ncomp; ++c) h << mins[size_t(b) * ncomp + c] << ',';
    h << '\n';
  }
  h << '\n' << nbox << ',' << ncomp << '\n';
  for (int b = 0; b < nbox; ++b) {
    for (int c = 0; c < ncomp; ++c) h << maxs[size_t(b) * ncomp + c] << ',';
    h << '\n';
  }
  if (!h) return io_fail("write failed: " + lev + "/" + mf + "_H");
  return CAMR_OK;
}

// The plotfile Header over nlev levels (refinement ratio 2 between them).
camr_status write_header(const std::string& root, const std::vector<std::string>& vnames,
                         const double prob_lo[3], const double prob_hi[3], double time,
                         const std::vector<LevelOut>& levels) {
  std::ofstream h(root + "/Header");
  if (!h) return io_fail("cannot write " + root + "/Header");
  const int nlev = int(levels.size());
  h << std::setprecision(17);
  h << "HyperCLaw-V1.1\n" << vnames.size() << '\n';
  for (const auto& v : vnames) h << v << '\n';
  h << 3 << '\n' << time << '\n' << nlev - 1 << '\n';
  for (int d = 0; d < 3; ++d) h << prob_lo[d] << ' ';
  h << '\n';
  for (int d = 0; d < 3; ++d) h << prob_hi[d] << ' ';
  h << '\n';
  for (int l = 0; l + 1 < nlev; ++l) h << 2 << ' ';
  h << '\n';
  for (const auto& L : levels) h << box_text(L.dom_lo, L.dom_hi) << ' ';
  h << '\n';
  for (const auto& L : levels) h << L.level_step << ' ';
  h << '\n';
  for (const auto& L : levels) {
    for (int d = 0; d < 3; ++d) h << L.dx[d] << ' ';
    h << '\n';
  }
  h << 0 << '\n' << "0\n";
  for (int l = 0; l < nlev; ++l) {
    const LevelOut& L = levels[size_t(l)];
    h << l << ' ' << L.nbox << ' ' << time << '\n' << L.level_step << '\n';
    for (int b = 0; b < L.nbox; ++b)
      for (int d = 0; d < 3; ++d) {
        const double lo = prob_lo[d] + L.boxes[6 * b + d] * L.dx[d];
        const double hi = prob_lo[d] + (L.boxes[6 * b + 3 + d] + 1) * L.dx[d];
        h << lo << ' ' << hi << '\n';
      }
    h << "Level_" << l << "/Cell\n";
  }
  if (!h) return io_fail("write failed: " + root + "/Header");
  return CAMR_OK;
}

camr_status check_names(int ncomp, const int* comps, const char* const* names,
                        std::vector<int>& cmap, std::vector<std::string>& vnames) {
  cmap.resize(size_t(ncomp));
  vnames.resize(size_t(ncomp));
  for (int c = 0; c < ncomp; ++c) {
    cmap[size_t(c)] = comps ? comps[c] : c;
    if (cmap[size_t(c)] < 0 || cmap[size_t(c)] >= CAMR_NVAR) return io_fail("component out of range");
    vnames[size_t(c)] = (names && names[c]) ? names[c] : kStateNames[cmap[size_t(c)]];
  }
  return CAMR_OK;
}

bool boxes_inside(int nbox, const int* boxes, const int dlo[3], const int dhi[3]);

// Header fields the readers check: variable count, dimension, time, finest
// level and the level steps.
camr_status read_header(const std::string& root, int ncomp, int* finest, double* time,
                        int steps[2]) {
  std::ifstream h(root + "/Header");
  if (!h) return io_fail("cannot read " + root + "/Header");
  std::string line;
  std::vector<std::string> lines;
  while (std::getline(h, line)) lines.push_back(line);
  if (lines.size() < 3 || lines[0] != "HyperCLaw-V1.1") return io_fail("unexpected plotfile header");
  const int nv = std::atoi(lines[1].c_str());
  if (nv != ncomp || lines.size() < size_t(nv) + 10) return io_fail("unexpected plotfile header");
  size_t i = 2 + size_t(nv);
  const int dim = std::atoi(lines[i].c_str());
  const double t = std::atof(lines[i + 1].c_str());
  *finest = std::atoi(lines[i + 2].c_str());
  if (dim != 3 || *finest < 0 || *finest > 1) return io_fail("only 3-D plotfiles of one or two levels are read");
  if (time) *time = t;
  std::istringstream st(lines[i + 7]);  // level steps
  for (int l = 0; l <= *finest; ++l) st >> steps[l];
  return CAMR_OK;
}

// A level's VisMF header: boxes (6 ints each), data files and offsets.
camr_status read_cell_h(const std::string& lev, int ncomp, std::vector<int>& bx,
                        std::vector<std::string>& files, std::vector<int64_t>& offs,
                        const std::string& mf = "Cell") {
  std::ifstream ch(lev + "/" + mf + "_H");
  if (!ch) return io_fail("cannot read " + lev + "/" + mf + "_H");
  int version = 0, how = 0, nc = 0, ngrow = 0;
  ch >> version >> how >> nc >> ngrow;
  if (nc != ncomp || ngrow != 0) return io_fail("unexpected Cell_H");
  char paren;
  int nbox = 0, zero = 0;
  ch >> paren >> nbox >> zero;
  // a count beyond any real BoxArray (a damaged header) is refused before
  // it sizes the box list
  constexpr int kMaxBoxes = 1 << 22;
  if (!ch || nbox < 0 || nbox > kMaxBoxes) return io_fail("bad box count in Cell_H");
  bx.assign(size_t(nbox) * 6, 0);
  for (int b = 0; b < nbox; ++b) {
    std::string tok;
    int lo[3], hi[3], ty[3];
    ch >> tok;  // "((lo0,lo1,lo2)"
    if (std::sscanf(tok.c_str(), "((%d,%d,%d)", &lo[0], &lo[1], &lo[2]) != 3)
      return io_fail("bad box in Cell_H");
    ch >> tok;
    if (std::sscanf(tok.c_str(), "(%d,%d,%d)", &hi[0], &hi[1], &hi[2]) != 3)
      return io_fail("bad box in Cell_H");
    ch >> tok;
    if (std::sscanf(tok.c_str(), "(%d,%d,%d))", &ty[0], &ty[1], &ty[2]) != 3)
      return io_fail("bad box in Cell_H");
    for (int d = 0; d < 3; ++d) {
      bx[size_t(6 * b + d)] = lo[d];
      bx[size_t(6 * b + 3 + d)] = hi[d];
    }
  }
  ch >> paren;
  int nfab = 0;
  ch >> nfab;
  if (nfab != nbox) return io_fail("unexpected FabOnDisk count");
  files.assign(size_t(nbox), "");
  offs.assign(size_t(nbox), 0);
  for (int b = 0; b < nbox; ++b) {
    std::string tag;
    ch >> tag >> files[size_t(b)] >> offs[size_t(b)];
    if (tag != "FabOnDisk:") return io_fail("bad FabOnDisk line");
  }
  return CAMR_OK;
}

// One FAB of box [lo, hi] into row(c, j, k)[i].
template <class Row>
camr_status read_fab(const std::string& file, int64_t off, const int lo[3], const int hi[3],
                     int ncomp, Row row) {
  std::FILE* f = std::fopen(file.c_str(), "rb");
  if (!f) return io_fail("cannot read " + file);
  if (std::fseek(f, long(off), SEEK_SET) != 0) {
    std::fclose(f);
    return io_fail("seek failed");
  }
  char line[512];
  if (!std::fgets(line, sizeof line, f) || std::strncmp(line, kFabFormat, std::strlen(kFabFormat))) {
    std::fclose(f);
    return io_fail("unexpected FAB header");
  }
  const int64_t bc = int64_t(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
  std::vector<double> buf(static_cast<size_t>(bc));
  for (int c = 0; c < ncomp; ++c) {
    if (std::fread(buf.data(), sizeof(double), size_t(bc), f) != size_t(bc)) {
      std::fclose(f);
      return io_fail("short FAB data");
    }
    int64_t t = 0;
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j) {
        double* r = row(c, j, k);
        for (int i = lo[0]; i <= hi[0]; ++i) r[i] = buf[size_t(t++)];
      }
  }
  std::fclose(f);
  return CAMR_OK;
}

// Level 0 into the domain-shaped state (first ncomp planes).
camr_status read_level0(const std::string& root, const camr_geom* geom, int ncomp, double* state) {
  int n[3];
  for (int d = 0; d < 3; ++d) n[d] = geom->dom_hi[d] - geom->dom_lo[d] + 1;
  const int64_t ncell = int64_t(n[0]) * n[1] * n[2];
  std::vector<int> bx;
  std::vector<std::string> files;
  std::vector<int64_t> offs;
  camr_status cs = read_cell_h(root + "/Level_0", ncomp, bx, files, offs);
  if (cs != CAMR_OK) return cs;
  const int nbox = int(files.size());
  if (!boxes_inside(nbox, bx.data(), geom->dom_lo, geom->dom_hi)) return io_fail("box outside domain");
  for (int b = 0; b < nbox; ++b) {
    cs = read_fab(root + "/Level_0/" + files[size_t(b)], offs[size_t(b)], &bx[size_t(6 * b)],
                  &bx[size_t(6 * b + 3)], ncomp, [&](int c, int j, int k) {
                    return state + int64_t(c) * ncell +
                           (int64_t(k - geom->dom_lo[2]) * n[1] + (j - geom->dom_lo[1])) * n[0] -
                           geom->dom_lo[0];
                  });
    if (cs != CAMR_OK) return cs;
  }
  return CAMR_OK;
}

bool boxes_inside(int nbox, const int* boxes, const int dlo[3], const int dhi[3]) {
  for (int b = 0; b < nbox; ++b)
    for (int d = 0; d < 3; ++d) {
      const int lo = boxes[6 * b + d], hi = boxes[6 * b + 3 + d];
      if (lo < dlo[d] || hi > dhi[d] || hi < lo) return false;
    }
  return true;
}

}  // namespace

extern "C" {

const char* camr_io_last_error(void) { return g_io_error.c_str(); }

camr_status camr_write_plotfile(const char* dir, const camr_geom* geom, const double prob_hi[3],
                                double time, int level_step, int nbox, const int* boxes,
                                const double* state, int ncomp, const int* comps,
                                const char* const* names) {
  g_io_error.clear();
  if (!dir || !geom || !prob_hi || nbox <= 0 || !boxes || !state || ncomp <= 0)
    return io_fail("invalid arguments");
  if (!host_little_endian()) return io_fail("big-endian hosts are not supported");
  std::vector<int> cmap;
  std::vector<std::string> vnames;
  camr_status cs = check_names(ncomp, comps, names, cmap, vnames);
  if (cs != CAMR_OK) return cs;
  if (!boxes_inside(nbox, boxes, geom->dom_lo, geom->dom_hi)) return io_fail("box outside the domain");
  int n[3];
  for (int d = 0; d < 3; ++d) n[d] = geom->dom_hi[d] - geom->dom_lo[d] + 1;
  const int64_t ncell = int64_t(n[0]) * n[1] * n[2];
  const std::string root(dir);
  if (!make_dir(root)) return io_fail("cannot create " + root);
  cs = write_level_files(root + "/Level_0", nbox, boxes, ncomp, [&](int, int c, int j, int k) {
    return state + int64_t(cmap[size_t(c)]) * ncell +
           (int64_t(k - geom->dom_lo[2]) * n[1] + (j - geom->dom_lo[1])) * n[0] - geom->dom_lo[0];
  });
  if (cs != CAMR_OK) return cs;
  LevelOut L0;
  for (int d = 0; d < 3; ++d) {
    L0.dom_lo[d] = geom->dom_lo[d];
    L0.dom_hi[d] = geom->dom_hi[d];
    L0.dx[d] = geom->dx[d];
  }
  L0.level_step = level_step;
  L0.nbox = nbox;
  L0.boxes = boxes;
  return write_header(root, vnames, geom->prob_lo, prob_hi, time, {L0});
}

camr_status camr_write_plotfile_amr(const char* dir, const camr_geom* geom, const double prob_hi[3],
                                    double time, const int level_step[2], int nbox0,
                                    const int* boxes0, const double* state0, int nbox1,
                                    const int* boxes1, const double* state1, int ncomp,
                                    const int* comps, const char* const* names) {
  g_io_error.clear();
  if (!dir || !geom || !prob_hi || !level_step || nbox0 <= 0 || !boxes0 || !state0 ||
      nbox1 < 0 || (nbox1 > 0 && (!boxes1 || !state1)) || ncomp <= 0)
    return io_fail("invalid arguments");
  if (!host_little_endian()) return io_fail("big-endian hosts are not supported");
  std::vector<int> cmap;
  std::vector<std::string> vnames;
  camr_status cs = check_names(ncomp, comps, names, cmap, vnames);
  if (cs != CAMR_OK) return cs;
  LevelOut L0, L1;
  for (int d = 0; d < 3; ++d) {
    L0.dom_lo[d] = geom->dom_lo[d];
    L0.dom_hi[d] = geom->dom_hi[d];
    L0.dx[d] = geom->dx[d];
    L1.dom_lo[d] = 2 * geom->dom_lo[d];
    L1.dom_hi[d] = 2 * geom->dom_hi[d] + 1;
    L1.dx[d] = geom->dx[d] / 2;
  }
  L0.level_step = level_step[0];
  L0.nbox = nbox0;
  L0.boxes = boxes0;
  L1.level_step = level_step[1];
  L1.nbox = nbox1;
  L1.boxes = boxes1;
  if (!boxes_inside(nbox0, boxes0, L0.dom_lo, L0.dom_hi) ||
      !boxes_inside(nbox1, boxes1, L1.dom_lo, L1.dom_hi))
    return io_fail("box outside the domain");
  int n[3];
  for (int d = 0; d < 3; ++d) n[d] = geom->dom_hi[d] - geom->dom_lo[d] + 1;
  const int64_t ncell = int64_t(n[0]) * n[1] * n[2];
  const std::string root(dir);
  if (!make_dir(root)) return io_fail("cannot create " + root);
  cs = write_level_files(root + "/Level_0", nbox0, boxes0, ncomp, [&](int, int c, int j, int k) {
    return state0 + int64_t(cmap[size_t(c)]) * ncell +
           (int64_t(k - geom->dom_lo[2]) * n[1] + (j - geom->dom_lo[1])) * n[0] - geom->dom_lo[0];
  });
  if (cs != CAMR_OK) return cs;
  // the fine boxes' states back to back, each (NVAR, nz, ny, nx) over its box
  std::vector<int64_t> base(size_t(nbox1) + 1, 0);
  for (int b = 0; b < nbox1; ++b) {
    const int* lo = boxes1 + 6 * b;
    const int* hi = boxes1 + 6 * b + 3;
    base[size_t(b) + 1] = base[size_t(b)] + int64_t(CAMR_NVAR) * (hi[0] - lo[0] + 1) *
                                                (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
  }
  if (nbox1 > 0) {
    cs = write_level_files(root + "/Level_1", nbox1, boxes1, ncomp, [&](int b, int c, int j, int k) {
      const int* lo = boxes1 + 6 * b;
      const int* hi = boxes1 + 6 * b + 3;
      const int64_t bx = hi[0] - lo[0] + 1, by = hi[1] - lo[1] + 1, bz = hi[2] - lo[2] + 1;
      return state1 + base[size_t(b)] + int64_t(cmap[size_t(c)]) * bx * by * bz +
             (int64_t(k - lo[2]) * by + (j - lo[1])) * bx - lo[0];
    });
    if (cs != CAMR_OK) return cs;
  }
  std::vector<LevelOut> levels{L0};
  if (nbox1 > 0) levels.push_back(L1);
  return write_header(root, vnames, geom->prob_lo, prob_hi, time, levels);
}

camr_status camr_read_plotfile(const char* dir, const camr_geom* geom, int ncomp,
                               double* state, double* time, int* level_step) {
  g_io_error.clear();
  if (!dir || !geom || ncomp <= 0 || !state) return io_fail("invalid arguments");
  // the state holds NVAR planes: more components would write past its end
  if (ncomp > CAMR_NVAR) return io_fail("ncomp exceeds NVAR");
  const std::string root(dir);
  int finest = 0;
  int steps[2] = {0, 0};
  camr_status cs = read_header(root, ncomp, &finest, time, steps);
  if (cs != CAMR_OK) return cs;
  if (finest != 0) return io_fail("only single-level 3-D plotfiles are read");
  if (level_step) *level_step = steps[0];
  return read_level0(root, geom, ncomp, state);
}

camr_status camr_read_plotfile_amr(const char* dir, const camr_geom* geom, int ncomp,
                                   double* state0, int nbox1, const int* boxes1,
                                   double* state1, double* time, int level_step[2]) {
  g_io_error.clear();
  if (!dir || !geom || ncomp <= 0 || !state0 || nbox1 < 0 || (nbox1 > 0 && (!boxes1 || !state1)))
    return io_fail("invalid arguments");
  // level-1 boxes lie NVAR planes apart in state1: more components would
  // write into the next box and past the end of the array
  if (ncomp > CAMR_NVAR) return io_fail("ncomp exceeds NVAR");
  const std::string root(dir);
  int finest = 0;
  int steps[2] = {0, 0};
  camr_status cs = read_header(root, ncomp, &finest, time, steps);
  if (cs != CAMR_OK) return cs;
  if (finest != (nbox1 > 0 ? 1 : 0)) return io_fail("level count differs from the hierarchy's");
  if (level_step) {
    level_step[0] = steps[0];
    level_step[1] = steps[1];
  }
  cs = read_level0(root, geom, ncomp, state0);
  if (cs != CAMR_OK || nbox1 == 0) return cs;
  // level 1: the same boxes, in the same order, as the hierarchy's
  std::vector<int> bx;
  std::vector<std::string> files;
  std::vector<int64_t> offs;
  cs = read_cell_h(root + "/Level_1", ncomp, bx, files, offs);
  if (cs != CAMR_OK) return cs;
  if (int(files.size()) != nbox1) return io_fail("fine box count differs from the hierarchy's");
  for (int k = 0; k < 6 * nbox1; ++k)
    if (bx[size_t(k)] != boxes1[k]) return io_fail("fine boxes differ from the hierarchy's");
  int64_t base = 0;
  for (int b = 0; b < nbox1; ++b) {
    const int* lo = boxes1 + 6 * b;
    const int* hi = boxes1 + 6 * b + 3;
    const int64_t bxn = hi[0] - lo[0] + 1, byn = hi[1] - lo[1] + 1, bzn = hi[2] - lo[2] + 1;
    double* dst = state1 + base;
    cs = read_fab(root + "/Level_1/" + files[size_t(b)], offs[size_t(b)], lo, hi, ncomp,
                  [&](int c, int j, int k) {
                    return dst + int64_t(c) * bxn * byn * bzn + (int64_t(k - lo[2]) * byn +
                                                                  (j - lo[1])) * bxn - lo[0];
                  });
    if (cs != CAMR_OK) return cs;
    base += int64_t(CAMR_NVAR) * bxn * byn * bzn;
  }
  return CAMR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Checkpoints: CAMR::checkPoint (Source/Utils/CAMR_io.cpp:45-60) is
// AmrLevel::checkPoint for each level inside Amr::checkPoint, plus the
// CPUtime file; restart (:23-43) reads them back.  The directory holds
//   Header          Amr's header: "CheckPointVersion_1.0", the dimension,
//                   the cumulative time, max and finest level, each level's
//                   Geometry, the refinement ratios, dt_level, dt_min,
//                   n_cycle, level_steps and level_count; then per level
//                   (AmrLevel::checkPoint) the level, its Geometry, the
//                   refinement ratio to the next level, the BoxArray, the
//                   number of state types (1) and the StateData record: the
//                   domain, the BoxArray, the old and new time intervals,
//                   the MultiFab count (1: no old data is dumped) and the
//                   relative name of the new data, Level_L/SD_0_New_MF;
//   Level_L/SD_0_New_MF_H, _D_00000   that MultiFab (VisMF, as plotfiles);
//   CPUtime         the elapsed CPU time, 15 digits.
// The text layout restates AMReX's stream formats (Geometry: coordinate
// system, offset and cell size; the real box; the index domain; the
// periodicity); AMReX itself is not present to read them, so this layout is
// not pinned by AMReX's own reader.  The library's reader reads back what
// the writer writes.
namespace {

const char* const kCheckpointVersion = "CheckPointVersion_1.0";
const char* const kStateMF = "SD_0_New_MF";

std::string geometry_text(const int dlo[3], const int dhi[3], const double dx[3],
                          const double plo[3], const double phi[3], const int periodic[3]) {
  std::ostringstream o;
  o << std::setprecision(17);
  o << "(0 (" << plo[0] << ',' << plo[1] << ',' << plo[2] << ")(" << dx[0] << ',' << dx[1] << ','
    << dx[2] << ") 1)";
  o << "(RealBox " << plo[0] << ' ' << phi[0] << ' ' << plo[1] << ' ' << phi[1] << ' ' << plo[2]
    << ' ' << phi[2] << " )";
  o << box_text(dlo, dhi) << " P(" << periodic[0] << ',' << periodic[1] << ',' << periodic[2]
    << ')';
  return o.str();
}

void boxarray_text(std::ostream& h, int nbox, const int* boxes) {
  h << '(' << nbox << " 0\n";
  for (int b = 0; b < nbox; ++b) h << box_text(boxes + 6 * b, boxes + 6 * b + 3) << '\n';
  h << ")\n";
}

// The state of level 0 (domain-shaped) or level 1 (boxes back to back) as
// the row function write_level_files takes.
struct LevelData {
  const camr_geom* geom;
  int nbox;
  const int* boxes;
  double* state;  // level 0: (NVAR, nz, ny, nx) of the domain; level 1: per box
  bool domain_shaped;
  std::vector<int64_t> base;
  void init() {
    base.assign(size_t(nbox) + 1, 0);
    for (int b = 0; b < nbox; ++b) {
      const int* lo = boxes + 6 * b;
      const int* hi = boxes + 6 * b + 3;
      base[size_t(b) + 1] = base[size_t(b)] + int64_t(CAMR_NVAR) * (hi[0] - lo[0] + 1) *
                                                  (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
    }
  }
  double* row(int b, int c, int j, int k) const {
    if (domain_shaped) {
      int n[3];
      for (int d = 0; d < 3; ++d) n[d] = geom->dom_hi[d] - geom->dom_lo[d] + 1;
      const int64_t ncell = int64_t(n[0]) * n[1] * n[2];
      return state + int64_t(c) * ncell +
             (int64_t(k - geom->dom_lo[2]) * n[1] + (j - geom->dom_lo[1])) * n[0] -
             geom->dom_lo[0];
    }
    const int* lo = boxes + 6 * b;
    const int* hi = boxes + 6 * b + 3;
    const int64_t bx = hi[0] - lo[0] + 1, by = hi[1] - lo[1] + 1, bz = hi[2] - lo[2] + 1;
    return state + base[size_t(b)] + int64_t(c) * bx * by * bz +
           (int64_t(k - lo[2]) * by + (j - lo[1])) * bx - lo[0];
  }
};

std::vector<std::string> read_lines(const std::string& path) {
  std::vector<std::string> lines;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) lines.push_back(line);
  return lines;
}

}  // namespace

extern "C" {

camr_status camr_write_checkpoint(const char* dir, const camr_geom* geom, const double prob_hi[3],
                                  const double time[2], const double dt[2],
                                  const int level_step[2], int nbox0, const int* boxes0,
                                  const double* state0, int nbox1, const int* boxes1,
                                  const double* state1, double cpu_time) {
  g_io_error.clear();
  if (!dir || !geom || !prob_hi || !time || !dt || !level_step || nbox0 <= 0 || !boxes0 ||
      !state0 || nbox1 < 0 || (nbox1 > 0 && (!boxes1 || !state1)))
    return io_fail("invalid arguments");
  if (!host_little_endian()) return io_fail("big-endian hosts are not supported");
  const int nlev = nbox1 > 0 ? 2 : 1;
  int dlo[2][3], dhi[2][3];
  double dxl[2][3];
  for (int d = 0; d < 3; ++d) {
    dlo[0][d] = geom->dom_lo[d];
    dhi[0][d] = geom->dom_hi[d];
    dxl[0][d] = geom->dx[d];
    dlo[1][d] = 2 * geom->dom_lo[d];
    dhi[1][d] = 2 * geom->dom_hi[d] + 1;
    dxl[1][d] = geom->dx[d] / 2;
  }
  if (!boxes_inside(nbox0, boxes0, dlo[0], dhi[0]) ||
      (nlev == 2 && !boxes_inside(nbox1, boxes1, dlo[1], dhi[1])))
    return io_fail("box outside the domain");
  const std::string root(dir);
  if (!make_dir(root)) return io_fail("cannot create " + root);
  const int nb[2] = {nbox0, nbox1};
  const int* bl[2] = {boxes0, boxes1};
  const double* sl[2] = {state0, state1};
  for (int l = 0; l < nlev; ++l) {
    LevelData D{geom, nb[l], bl[l], const_cast<double*>(sl[l]), l == 0, {}};
    D.init();
    camr_status cs = write_level_files(
        root + "/Level_" + std::to_string(l), nb[l], bl[l], CAMR_NVAR,
        [&](int b, int c, int j, int k) { return D.row(b, c, j, k); }, kStateMF);
    if (cs != CAMR_OK) return cs;
  }
  std::ofstream h(root + "/Header");
  if (!h) return io_fail("cannot write " + root + "/Header");
  h << std::setprecision(17);
  h << kCheckpointVersion << '\n' << 3 << '\n' << time[0] << '\n' << nlev - 1 << '\n'
    << nlev - 1 << '\n';
  std::string gtext[2];
  for (int l = 0; l < nlev; ++l) {
    gtext[l] = geometry_text(dlo[l], dhi[l], dxl[l], geom->prob_lo, prob_hi, geom->is_periodic);
    h << gtext[l] << ' ';
  }
  h << '\n';
  for (int l = 0; l + 1 < nlev; ++l) h << "(2,2,2) ";
  h << '\n';
  for (int l = 0; l < nlev; ++l) h << dt[l] << ' ';  // dt_level
  h << '\n';
  for (int l = 0; l < nlev; ++l) h << dt[l] << ' ';  // dt_min
  h << '\n';
  for (int l = 0; l < nlev; ++l) h << (l == 0 ? 1 : 2) << ' ';  // n_cycle
  h << '\n';
  for (int l = 0; l < nlev; ++l) h << level_step[l] << ' ';
  h << '\n';
  for (int l = 0; l < nlev; ++l) h << 0 << ' ';  // level_count (steps since regrid)
  h << '\n';
  for (int l = 0; l < nlev; ++l) {
    h << l << '\n' << gtext[l] << '\n' << (l + 1 < nlev ? "(2,2,2)" : "(1,1,1)") << '\n';
    boxarray_text(h, nb[l], bl[l]);
    h << 1 << '\n';
    // StateData::checkPoint
    h << box_text(dlo[l], dhi[l]) << '\n';
    boxarray_text(h, nb[l], bl[l]);
    h << time[l] - dt[l] << '\n' << time[l] - dt[l] << '\n' << time[l] << '\n' << time[l] << '\n';
    h << 1 << '\n' << "Level_" << l << '/' << kStateMF << '\n';
  }
  if (!h) return io_fail("write failed: " + root + "/Header");
  std::ofstream cpu(root + "/CPUtime");
  cpu << std::setprecision(15) << cpu_time;
  if (!cpu) return io_fail("write failed: " + root + "/CPUtime");
  return CAMR_OK;
}

camr_status camr_read_checkpoint(const char* dir, const camr_geom* geom, double time[2],
                                 double dt[2], int level_step[2], double* state0, int nbox1,
                                 const int* boxes1, double* state1) {
  g_io_error.clear();
  if (!dir || !geom || !time || !dt || !level_step || !state0 || nbox1 < 0 ||
      (nbox1 > 0 && (!boxes1 || !state1)))
    return io_fail("invalid arguments");
  const std::string root(dir);
  const std::vector<std::string> L = read_lines(root + "/Header");
  if (L.size() < 12 || L[0] != kCheckpointVersion || std::atoi(L[1].c_str()) != 3)
    return io_fail("not a 3-D checkpoint of this layout");
  const int finest = std::atoi(L[4].c_str());
  if (finest != (nbox1 > 0 ? 1 : 0)) return io_fail("level count differs from the hierarchy's");
  const int nlev = finest + 1;
  // lines: 5 geometries, 6 ratios, 7 dt_level, 8 dt_min, 9 n_cycle, 10 level_steps
  {
    std::istringstream a(L[7]), b(L[10]);
    for (int l = 0; l < nlev; ++l) a >> dt[l];
    for (int l = 0; l < nlev; ++l) b >> level_step[l];
  }
  // per level: the StateData record's new time (the line after the old
  // interval) -- find each "Level_L/SD_0_New_MF" line and read back 2 lines
  for (int l = 0; l < nlev; ++l) {
    const std::string tag = "Level_" + std::to_string(l) + "/" + kStateMF;
    size_t at = 0;
    while (at < L.size() && L[at] != tag) ++at;
    if (at == L.size() || at < 3) return io_fail("no state record for level " + std::to_string(l));
    time[l] = std::atof(L[at - 2].c_str());
  }
  for (int l = 0; l < nlev; ++l) {
    std::vector<int> bx;
    std::vector<std::string> files;
    std::vector<int64_t> offs;
    const std::string lev = root + "/Level_" + std::to_string(l);
    camr_status cs = read_cell_h(lev, CAMR_NVAR, bx, files, offs, kStateMF);
    if (cs != CAMR_OK) return cs;
    const int nbox = int(files.size());
    if (l == 0) {
      if (!boxes_inside(nbox, bx.data(), geom->dom_lo, geom->dom_hi))
        return io_fail("box outside domain");
    } else {
      if (nbox != nbox1) return io_fail("fine box count differs from the hierarchy's");
      for (int k = 0; k < 6 * nbox1; ++k)
        if (bx[size_t(k)] != boxes1[k]) return io_fail("fine boxes differ from the hierarchy's");
    }
    LevelData D{geom, nbox, l == 0 ? bx.data() : boxes1, l == 0 ? state0 : state1, l == 0, {}};
    D.init();
    for (int b = 0; b < nbox; ++b) {
      cs = read_fab(lev + "/" + files[size_t(b)], offs[size_t(b)], &bx[size_t(6 * b)],
                    &bx[size_t(6 * b + 3)], CAMR_NVAR,
                    [&](int c, int j, int k) { return D.row(b, c, j, k); });
      if (cs != CAMR_OK) return cs;
    }
  }
  return CAMR_OK;
}

}  // extern "C"
