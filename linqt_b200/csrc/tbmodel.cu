// Operator builder, host side: LinQT's utilities/wannier2sparse model files, unit-cell
// operators and the supercell plan the device kernels (supercell.cu) expand.
//
// The reference keeps hoppings in a std::multimap keyed by the text tag "cx cy cz e0 e1 "
// (include/hopping_list.hpp:163-171, 226), so every list is iterated in string order of
// that tag, equal tags in insertion order.  The order matters twice: it is the order in
// which duplicate matrix entries are summed (Eigen's setFromTriplets, a left fold in
// triplet order, src/hopping_list.cpp:245-257) and the order of the torque's on-site sums.
// Lists here are kept in that order (ordered()), and the complex arithmetic is written in
// the same form as the reference's so that values agree to the bit.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <functional>
#include <map>
#include <numeric>
#include <sstream>
#include <thread>

#include "w2s.cuh"

namespace linqt {
namespace w2s {

namespace {

const char *const kAvailOps[18] = {"VX",   "VY",   "VZ",   "VXSX", "VXSY", "VXSZ", "VYSX", "VYSY", "VYSZ",
                                   "VZSX", "VZSY", "VZSZ", "SX",   "SY",   "SZ",   "TX",   "TY",   "TZ"};

int op_index(const std::string &op) {
  for (int i = 0; i < 18; ++i)
    if (op == kAvailOps[i]) return i;
  return -1;
}

std::string tag_of(const Hop &h) {
  std::string t;
  for (int x : h.cell) t += std::to_string(x) + " ";
  t += std::to_string(h.e0) + " " + std::to_string(h.e1) + " ";
  return t;
}

// insertion order -> the reference's iteration order (stable sort by tag)
std::vector<Hop> ordered(const std::vector<Hop> &in) {
  std::vector<std::pair<std::string, size_t>> t(in.size());
  for (size_t i = 0; i < in.size(); ++i) t[i] = {tag_of(in[i]), i};
  std::stable_sort(t.begin(), t.end(), [](const std::pair<std::string, size_t> &a,
                                          const std::pair<std::string, size_t> &b) { return a.first < b.first; });
  std::vector<Hop> out;
  out.reserve(in.size());
  for (auto &e : t) out.push_back(in[e.second]);
  return out;
}

double volume(const double uc[3][3]) {  // tbmodel.cpp:492-498
  return std::fabs((uc[0][1] * uc[1][2] - uc[1][1] * uc[0][2]) * uc[2][0] +
                   (uc[0][2] * uc[1][0] - uc[0][0] * uc[1][2]) * uc[2][1] +
                   (uc[0][0] * uc[1][1] - uc[0][1] * uc[1][0]) * uc[2][2]);
}

int parse_int_line(const std::string &line, const std::string &what) {
  try {
    return std::stoi(line);
  } catch (const std::exception &) {
    fail(LINQT_ERR_INVALID, "cannot read " + what + " from \"" + line + "\"");
  }
}

// wannier_parser.cpp:45-84 + hopping_list.cpp:114-155: line 0 is a comment, then
// num_wann, nrpts, nrpts/15 + 1 lines of degeneracies, then one hopping per line
// "Rx Ry Rz m n Re Im" (orbitals 1-based).  Hoppings with |t| <= 1e-10 of the mean |t|
// are dropped.  Blank lines are skipped (the reference parses them from uninitialised
// values).
std::vector<Hop> read_hr(const std::string &path, int &num_wann) {
  std::ifstream f(path);
  LQ_REQUIRE(f.is_open(), "cannot open " + path);
  std::string line;
  int nrpts = 0;
  std::vector<Hop> parsed;
  for (int counter = 0; std::getline(f, line); counter++) {
    if (counter == 0) continue;
    if (counter == 1) {
      num_wann = parse_int_line(line, "num_wann");
      LQ_REQUIRE(num_wann > 0, path + ": num_wann must be positive");
      continue;
    }
    if (counter == 2) {
      nrpts = parse_int_line(line, "nrpts");
      LQ_REQUIRE(nrpts > 0, path + ": nrpts must be positive");
      continue;
    }
    if (counter == 3) {
      for (int k = 0; k < nrpts / 15; ++k) {
        std::getline(f, line);
        counter++;
      }
      continue;
    }
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    std::istringstream ss(line);
    Hop h;
    double re = 0, im = 0;
    ss >> h.cell[0] >> h.cell[1] >> h.cell[2] >> h.e0 >> h.e1 >> re >> im;
    LQ_REQUIRE(!ss.fail(), path + ": malformed hopping line " + std::to_string(counter + 1) + ": \"" + line + "\"");
    h.e0 -= 1;
    h.e1 -= 1;
    LQ_REQUIRE(h.e0 >= 0 && h.e0 < num_wann && h.e1 >= 0 && h.e1 < num_wann,
               path + ": orbital index out of range on line " + std::to_string(counter + 1));
    h.v = cplx(re, im);
    parsed.push_back(h);
  }
  LQ_REQUIRE(num_wann > 0, path + ": missing header");
  double avg = 0;
  for (auto &h : parsed) avg += std::sqrt(std::norm(h.v));
  avg /= (double)parsed.size();
  std::vector<Hop> kept;
  for (auto &h : parsed)
    if (std::sqrt(std::norm(h.v)) / avg > 1e-10) kept.push_back(h);
  return ordered(kept);
}

void require_geometry(const Model &m) {
  LQ_REQUIRE((int)m.pos.size() == m.num_wann, "the .xyz file lists " + std::to_string(m.pos.size()) +
                                                  " orbitals, the _hr.dat file " + std::to_string(m.num_wann));
  LQ_REQUIRE(volume(m.lat) > 0, "the unit cell (.uc) has zero volume");
}

void require_spinful(const Model &m) {
  LQ_REQUIRE(m.num_wann % 2 == 0, "spin operators need an even number of orbitals (spin up block first)");
}

// tbmodel.cpp:92-126: t * (0, -dx_dir), dx = pos[e1] - pos[e0] + R . lattice, or 0 when
// |dx_dir| <= 1e-10 of the cube root of the cell volume.  Same tags, same order.
std::vector<Hop> currents(const Model &m, int dir) {
  require_geometry(m);
  const double av_length = std::pow(volume(m.lat), 1.0 / 3.0);
  std::vector<Hop> out = m.hops;
  for (auto &h : out) {
    std::array<double, 3> diff = m.pos[h.e1];
    for (int i = 0; i < 3; ++i) diff[i] += -m.pos[h.e0][i];
    std::array<double, 3> displ = {0, 0, 0};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) displ[i] += h.cell[j] * m.lat[j][i];
    for (int i = 0; i < 3; ++i) diff[i] += displ[i];
    if (std::fabs(diff[dir]) / av_length > 1E-10)
      h.v *= cplx(0.0, -diff[dir]);
    else
      h.v *= cplx(0.0, 0.0);
  }
  return out;
}

using Dense = std::vector<std::vector<cplx>>;

// tbmodel.cpp:64-90: every (i, j) entry of an on-site matrix, zeros included
std::vector<Hop> density(const Model &m, const Dense &op) {
  require_geometry(m);
  std::vector<Hop> out;
  const int n = m.num_wann;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) out.push_back(Hop{{0, 0, 0}, i, j, op[i][j]});
  return ordered(out);
}

// tbmodel.cpp:362-380: a 2x2 matrix (row major) on the spin pair (io, io + n/2) of every orbital
Dense spinorial(const Model &m, const std::array<cplx, 4> &op) {
  require_spinful(m);
  const int tot = m.num_wann, od = tot / 2;
  Dense s(tot, std::vector<cplx>(tot, cplx(0.0)));
  for (int io = 0; io < od; io++)
    for (int si = 0; si < 2; si++)
      for (int sj = 0; sj < 2; sj++) s[si * od + io][sj * od + io] = op[si * 2 + sj];
  return s;
}

std::array<cplx, 4> spin_elems(double theta, double phi) {  // tbmodel.cpp:144-148
  const cplx I(0, 1);
  return {cplx(std::cos(theta)), -std::sin(theta) * std::exp(-I * phi), std::sin(theta) * std::exp(I * phi),
          cplx(-std::cos(theta))};
}

// tbmodel.cpp:393-440: exchange field J of each orbital from the constant on-site block H00
Dense torque(const Model &m, double theta, double phi) {
  require_geometry(m);
  require_spinful(m);
  const cplx I(0, 1);
  const int tot = m.num_wann, od = tot / 2;
  Dense H00(tot, std::vector<cplx>(tot, cplx(0.0)));
  std::vector<Hop> onsite;
  for (auto &h : m.hops)
    if (h.cell[0] == 0 && h.cell[1] == 0 && h.cell[2] == 0) onsite.push_back(h);
  for (auto &h : ordered(onsite)) H00[h.e0][h.e1] += h.v;
  Dense Tu(tot, std::vector<cplx>(tot, cplx(0.0)));
  for (int io = 0; io < od; io++) {
    const int i = io, j = od + io;
    const cplx J00 = 0.5 * (H00[i][i] - H00[j][j]);
    const cplx J01 = 0.5 * (H00[i][j] + std::conj(H00[j][i]));
    const double J[3] = {J01.real(), -J01.imag(), J00.real()};
    Tu[i][i] = 1.0 * std::sin(theta) * (J[1] * std::cos(phi) - J[0] * std::sin(phi));
    Tu[j][j] = -1.0 * std::sin(theta) * (J[1] * std::cos(phi) - J[0] * std::sin(phi));
    Tu[i][j] = (-I * J[0] - J[1]) * std::cos(theta) + J[2] * std::sin(theta) * (I * std::cos(phi) + std::sin(phi));
    Tu[j][i] = std::conj(Tu[i][j]);
  }
  return Tu;
}

// tbmodel.cpp:162-212: the current of direction dir times the spin along (theta, phi)
std::vector<Hop> spin_currents(const Model &m, int dir, double theta, double phi) {
  require_spinful(m);
  const cplx I(0.0, 1.0);
  const int ns = m.num_wann / 2;
  auto chg = [ns](const Hop &h, int s0, int s1) {
    Hop o = h;
    o.e0 = h.e0 % ns + s0 * ns;
    o.e1 = h.e1 % ns + s1 * ns;
    return o;
  };
  std::vector<Hop> out;
  for (const Hop &h : currents(m, dir)) {
    const int is0 = h.e0 / ns, is1 = h.e1 / ns;
    const double sz = 1.0 - 2.0 * is0;
    if (is0 == is1) {
      const double s_uu = sz * std::cos(theta);
      const cplx s_ud = 0.5 * std::sin(theta) * std::exp(-I * phi);
      if (std::norm(s_uu) > 1e-5) {
        Hop o = chg(h, is0, is0);
        o.v *= cplx(s_uu);
        out.push_back(o);
      }
      if (std::norm(s_ud) > 1e-5) {
        Hop ud = chg(h, 0, 1), du = chg(h, 1, 0);
        ud.v *= s_ud;
        du.v *= std::conj(s_ud);
        out.push_back(ud);
        out.push_back(du);
      }
    } else {
      const cplx s_uu = 0.5 * std::sin(theta) * std::exp(sz * I * phi);
      if (std::norm(s_uu) > 1e-5) {
        Hop uu = chg(h, 0, 0), dd = chg(h, 1, 1);
        uu.v *= s_uu;
        dd.v *= s_uu;
        out.push_back(uu);
        out.push_back(dd);
      }
    }
  }
  return ordered(out);
}

void angles(char d, double &theta, double &phi) {  // tbmodel.cpp:218-224
  theta = d == 'Z' ? 0.0 * M_PI : 0.5 * M_PI;
  phi = d == 'Y' ? 0.5 * M_PI : 0.0 * M_PI;
}

int mod(int x, int d) {
  const int r = x % d;
  return r < 0 ? r + d : r;
}

}  // namespace

Model load_model(const std::string &label) {
  Model m;
  {  // wannier_parser.cpp:86-104
    std::ifstream f(label + ".xyz");
    LQ_REQUIRE(f.is_open(), "cannot open " + label + ".xyz");
    int n = 0;
    f >> n;
    LQ_REQUIRE(!f.fail() && n > 0, label + ".xyz: bad orbital count");
    for (int i = 0; i < n; ++i) {
      std::string l;
      std::array<double, 3> p;
      f >> l >> p[0] >> p[1] >> p[2];
      LQ_REQUIRE(!f.fail(), label + ".xyz: malformed orbital " + std::to_string(i + 1));
      m.labels.push_back(l);
      m.pos.push_back(p);
    }
  }
  {  // wannier_parser.cpp:106-117
    std::ifstream f(label + ".uc");
    LQ_REQUIRE(f.is_open(), "cannot open " + label + ".uc");
    for (auto &v : m.lat)
      for (double &x : v) f >> x;
    LQ_REQUIRE(!f.fail(), label + ".uc: expected 3 lattice vectors");
  }
  m.hops = read_hr(label + "_hr.dat", m.num_wann);
  // tbmodel.cpp:26-36: a LABEL.stdis file adds random hoppings drawn from a generator seeded
  // by std::random_device; that path is not reproduced
  std::ifstream dis(label + ".stdis");
  if (dis.is_open())
    fail(LINQT_ERR_UNSUPPORTED, label + ".stdis: static disorder files are not supported by the operator builder");
  return m;
}

bool is_builtin_op(const std::string &op) { return op == "HAM" || op_index(op) >= 0; }

std::vector<Hop> operator_list(const Model &m, const std::string &op) {
  if (op == "HAM") return m.hops;
  const int k = op_index(op);
  double theta = 0, phi = 0;
  if (k >= 0 && k < 3) return currents(m, op[1] - 'X');
  if (k >= 3 && k < 12) {
    angles(op.back(), theta, phi);
    return spin_currents(m, op[1] - 'X', theta, phi);
  }
  if (k >= 12 && k < 15) {
    angles(op.back(), theta, phi);
    return density(m, spinorial(m, spin_elems(theta, phi)));
  }
  if (k >= 15) {
    angles(op.back(), theta, phi);
    return density(m, torque(m, theta, phi));
  }
  // tbmodel.cpp:331-354: NAME.OP in the working directory: a type word, then 4 complex
  // numbers (re im), the spin matrix in row-major order
  std::ifstream f(op + ".OP");
  LQ_REQUIRE(f.good(), "unknown operator \"" + op + "\" (and no " + op + ".OP file)");
  std::string type;
  f >> type;
  std::array<cplx, 4> el;
  for (auto &e : el) {
    double re = 0, im = 0;
    f >> re >> im;
    e = cplx(re, im);
  }
  LQ_REQUIRE(!f.fail(), op + ".OP: expected a type and 4 complex numbers");
  return density(m, spinorial(m, el));
}

// hopping_list.cpp:158-257 restated per row: in the supercell, hopping (R, e0 -> e1) of the
// cell shift s lands on row (s, e0), column (s + R mod D, e1); two hoppings of the same
// row meet on one column exactly when their R agree mod D, whatever s.  So the entries of
// every row of orbital e0 are the keys (R mod D, e1), each the left fold, in list order, of
// the hoppings that map to it and pass the |v| > 1e-10 mean|v| filter.  The mean runs over
// the unit-cell list here; the reference sums the same values replicated over the cells in
// another order, which can only move an entry whose ratio is within rounding of 1e-10.
Plan make_plan(const std::vector<Hop> &uc, int wbb, const int dims[3]) {
  Plan p;
  p.wbb = wbb;
  for (int d = 0; d < 3; ++d) {
    LQ_REQUIRE(dims[d] > 0, "supercell dimensions must be positive");
    p.dims[d] = dims[d];
  }
  LQ_REQUIRE(wbb < 65536, "more than 65535 orbitals per cell");
  p.ncells = (long)dims[0] * dims[1] * dims[2];
  p.n = p.ncells * wbb;
  LQ_REQUIRE(p.n <= 0x7fffffffL, "the supercell has more than 2^31-1 orbitals");
  double avg = 0;
  for (auto &h : uc) avg += std::sqrt(std::norm(h.v));
  avg /= (double)uc.size();
  std::map<std::array<int, 5>, cplx> keys;
  for (auto &h : uc) {
    if (!(std::sqrt(std::norm(h.v)) / avg > 1E-10)) continue;
    LQ_REQUIRE(h.e0 >= 0 && h.e0 < wbb && h.e1 >= 0 && h.e1 < wbb, "orbital index out of range");
    const std::array<int, 5> k = {h.e0, mod(h.cell[2], dims[2]), mod(h.cell[1], dims[1]), mod(h.cell[0], dims[0]),
                                  h.e1};
    auto f = keys.find(k);
    if (f == keys.end())
      keys.emplace(k, h.v);
    else
      f->second = f->second + h.v;
  }
  LQ_REQUIRE(keys.size() < 0x7fffffffUL, "too many distinct entries per cell");
  p.grp_key0.assign(wbb + 1, 0);
  p.grp_z0.assign(wbb + 1, 0);
  auto it = keys.begin();
  for (int g = 0; g < wbb; ++g) {
    p.grp_key0[g] = p.keys();
    p.grp_z0[g] = (int)p.zn.size();
    const int g0 = p.keys();
    int zs = 0, ys = 0, xs = 0;  // first key of the current z / y / x run
    bool first = true;
    for (; it != keys.end() && it->first[0] == g; ++it) {
      const auto &k = it->first;
      const int K = p.keys();
      const bool nz = first || p.zn.back().val != k[1];
      const bool ny = nz || p.yn.back().val != k[2];
      const bool nx = ny || p.xn.back().val != k[3];
      first = false;
      if (nz) {
        zs = K;
        p.zn.push_back(Node{k[1], K - g0, 0, (int)p.yn.size(), 0, g});
      }
      if (ny) {
        ys = K;
        p.yn.push_back(Node{k[2], K - zs, 0, (int)p.xn.size(), 0, (int)p.zn.size() - 1});
        p.zn.back().nc++;
      }
      if (nx) {
        xs = K;
        p.xn.push_back(Node{k[3], K - ys, 0, K, 0, (int)p.yn.size() - 1});
        p.yn.back().nc++;
      }
      p.zn.back().size++;
      p.yn.back().size++;
      p.xn.back().size++;
      p.kz.push_back((int)p.zn.size() - 1);
      p.ky.push_back((int)p.yn.size() - 1);
      p.kx.push_back((int)p.xn.size() - 1);
      p.kleaf.push_back(K - xs);
      p.ko1.push_back(k[4]);
      p.kgrp.push_back(g);
      p.kval.push_back(make_double2(it->second.real(), it->second.imag()));
      p.kpack.push_back(make_int4(p.kz.back(), p.ky.back(), p.kx.back(), p.kleaf.back()));
      p.kgo.push_back(g << 16 | k[4]);
    }
  }
  p.grp_key0[wbb] = p.keys();
  p.grp_z0[wbb] = (int)p.zn.size();
  return p;
}

// hopping_list.cpp:260-282 with std::ostream's defaults (%g, 6 significant digits): the
// header "n nnz", then one line of "re im " pairs, one of "col ", one of "rowptr ".  The
// lines are formatted by all host threads in slices and written in order.
void write_csr_text(const std::string &path, long n, const std::vector<int> &rowptr, const std::vector<int> &col,
                    const std::vector<double2> &val) {
  std::FILE *f = std::fopen(path.c_str(), "w");
  LQ_REQUIRE(f, "cannot write " + path);
  const long nnz = (long)col.size();
  std::fprintf(f, "%ld %ld\n", n, nnz);
  const int nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  auto emit = [&](long count, const std::function<void(std::string &, long)> &fmt) {
    const long slice = 1L << 16;
    for (long base = 0; base < count; base += slice * nt) {
      std::vector<std::string> out(nt);
      std::vector<std::thread> th;
      for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
          const long lo = base + t * slice, hi = std::min(count, lo + slice);
          for (long k = lo; k < hi; ++k) fmt(out[t], k);
        });
      for (auto &x : th) x.join();
      for (auto &s : out) std::fwrite(s.data(), 1, s.size(), f);
    }
    std::fputc('\n', f);
  };
  emit(nnz, [&](std::string &s, long k) {
    char b[64];
    const int w = std::snprintf(b, sizeof b, "%g %g ", val[k].x, val[k].y);
    s.append(b, w);
  });
  emit(nnz, [&](std::string &s, long k) {
    char b[16];
    const int w = std::snprintf(b, sizeof b, "%d ", col[k]);
    s.append(b, w);
  });
  emit(n + 1, [&](std::string &s, long k) {
    char b[16];
    const int w = std::snprintf(b, sizeof b, "%d ", rowptr[k]);
    s.append(b, w);
  });
  LQ_REQUIRE(std::fclose(f) == 0, "error writing " + path);
}

}  // namespace w2s
}  // namespace linqt
