// CPU FP64 oracle (test infrastructure only; see oracle.h for the contract).
// Every function names the reference file:line it restates.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <unordered_map>
#include <vector>

namespace {

constexpr int BS = 8;
constexpr int BN = 512;

enum { K_SAME = 0, K_BOUNDARY = 1, K_COARSER = 2, K_FINER = 3 };
enum { BC_FREESPACE = 0, BC_PERIODIC = 1, BC_WALL = 2 };

inline int tan1(int d) { return d == 0 ? 1 : 0; }
inline int tan2(int d) { return d == 2 ? 1 : 2; }
inline int cell(int x, int y, int z) { return x + BS * y + BS * BS * z; }

// Sum of term(i), i < n, in an order that does not depend on the thread
// count or on scheduling: fixed chunks summed in parallel, chunk sums added
// serially in chunk order.  (An OpenMP reduction combines the threads'
// partials in arrival order, so its last bits vary from run to run, and
// BiCGSTAB's iteration count with them where the restart test or the
// stopping test is close.)
template <class F>
double det_sum(int64_t n, F term) {
  constexpr int64_t C = 4096;
  const int64_t nc = (n + C - 1) / C;
  std::vector<double> part(size_t(std::max<int64_t>(nc, 1)), 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    double s = 0;
    const int64_t e = std::min(n, (c + 1) * C);
    for (int64_t i = c * C; i < e; ++i) s += term(i);
    part[size_t(c)] = s;
  }
  double s = 0;
  for (int64_t c = 0; c < nc; ++c) s += part[size_t(c)];
  return s;
}

}  // namespace

struct orc_mesh {
  int nb = 0;
  int bpd[3] = {1, 1, 1};
  int level_max = 1;
  int bc[3] = {0, 0, 0};
  double h0 = 0, hmin = 0;
  std::vector<int> level;
  std::vector<std::array<int, 3>> idx;
  std::vector<double> h;
  std::vector<std::array<int, 6>> kind;
  std::vector<std::array<std::array<int, 4>, 6>> nbr;
  int mean_block = -1;
  std::map<std::array<int, 4>, int> lookup;  // independent of the product's hash table
  struct CSR {
    std::vector<int64_t> rowptr, col;
    std::vector<double> val;
  };
  CSR csr[4];  // assembled operator per mean-constraint mode (filled on first use)

  int find(int l, int i, int j, int k) const {
    auto it = lookup.find({l, i, j, k});
    return it == lookup.end() ? -1 : it->second;
  }
  // Znei lookup with periodic wrap (Cubism BlockInfo::Znei semantics).
  bool nei_index(int b, int d, int side, int n[3]) const {
    const int l = level[b];
    for (int e = 0; e < 3; ++e) n[e] = idx[b][e];
    n[d] += side ? 1 : -1;
    const int N = bpd[d] << l;
    if (n[d] < 0 || n[d] >= N) {
      if (bc[d] != BC_PERIODIC) return false;
      n[d] = (n[d] + N) % N;
    }
    return true;
  }
};

extern "C" orc_mesh* orc_mesh_create(int nb, const int32_t* level, const int32_t* index,
                                     const int32_t* bpd, int level_max, const int32_t* bc,
                                     double extent) {
  orc_mesh* m = new orc_mesh();
  m->nb = nb;
  for (int d = 0; d < 3; ++d) {
    m->bpd[d] = bpd[d];
    m->bc[d] = bc[d];
  }
  m->level_max = level_max;
  // SimulationData.cpp:141-165
  const int aux = 1 << (level_max - 1);
  const double nfe[3] = {double(bpd[0]) * aux * BS, double(bpd[1]) * aux * BS,
                         double(bpd[2]) * aux * BS};
  const double maxbpd = std::max({nfe[0], nfe[1], nfe[2]});
  const double ex0 = (nfe[0] / maxbpd) * extent;
  m->hmin = ex0 / nfe[0];
  m->h0 = ex0 * aux / nfe[0];
  m->level.resize(nb);
  m->idx.resize(nb);
  m->h.resize(nb);
  for (int b = 0; b < nb; ++b) {
    m->level[b] = level[b];
    m->idx[b] = {index[3 * b], index[3 * b + 1], index[3 * b + 2]};
    m->h[b] = std::ldexp(m->h0, -level[b]);
    if (!m->lookup.emplace(std::array<int, 4>{level[b], index[3 * b], index[3 * b + 1],
                                              index[3 * b + 2]},
                           b)
             .second) {
      delete m;
      return nullptr;
    }
    if (index[3 * b] == 0 && index[3 * b + 1] == 0 && index[3 * b + 2] == 0) m->mean_block = b;
  }
  m->kind.resize(nb);
  m->nbr.resize(nb);
  for (int b = 0; b < nb; ++b) {
    const int l = m->level[b];
    for (int d = 0; d < 3; ++d)
      for (int side = 0; side < 2; ++side) {
        const int f = 2 * d + side;
        m->nbr[b][f] = {-1, -1, -1, -1};
        int n[3];
        if (!m->nei_index(b, d, side, n)) {
          m->kind[b][f] = K_BOUNDARY;
          m->nbr[b][f][0] = m->bc[d];
          continue;
        }
        int id = m->find(l, n[0], n[1], n[2]);
        if (id >= 0) {
          m->kind[b][f] = K_SAME;
          m->nbr[b][f][0] = id;
          continue;
        }
        id = l > 0 ? m->find(l - 1, n[0] / 2, n[1] / 2, n[2] / 2) : -1;
        if (id >= 0) {
          m->kind[b][f] = K_COARSER;
          m->nbr[b][f][0] = id;
          continue;
        }
        m->kind[b][f] = K_FINER;
        const int t1 = tan1(d), t2 = tan2(d);
        for (int bb = 0; bb < 2; ++bb)
          for (int aa = 0; aa < 2; ++aa) {
            int c[3];
            c[d] = 2 * n[d] + (side == 0 ? 1 : 0);
            c[t1] = 2 * n[t1] + aa;
            c[t2] = 2 * n[t2] + bb;
            const int ch = m->find(l + 1, c[0], c[1], c[2]);
            if (ch < 0) {
              delete m;
              return nullptr;
            }
            m->nbr[b][f][aa + 2 * bb] = ch;
          }
      }
  }
  return m;
}

extern "C" void orc_mesh_destroy(orc_mesh* m) { delete m; }
extern "C" int orc_mesh_nb(const orc_mesh* m) { return m->nb; }
extern "C" double orc_mesh_h(const orc_mesh* m, int b) { return m->h[b]; }
extern "C" double orc_mesh_hmin(const orc_mesh* m) { return m->hmin; }
extern "C" void orc_mesh_faces(const orc_mesh* m, int32_t* kinds, int32_t* nbrs) {
  for (int b = 0; b < m->nb; ++b)
    for (int f = 0; f < 6; ++f) {
      kinds[6 * b + f] = m->kind[b][f];
      for (int q = 0; q < 4; ++q) nbrs[24 * b + 4 * f + q] = m->nbr[b][f][q];
    }
}

// ============================================================================
// Poisson matrix rows, PoissonSolverExp.cpp:112-373 and PoissonSolverExp.h:63-478
// ============================================================================
namespace {

using Row = std::map<int64_t, double>;  // SpRowInfo::mapColVal accumulates per column

struct FaceIdx {
  // Indexer for the face normal to d on side `side` of a block (the reference's
  // [XYZ]{min,max}Indexer), plus the Taylor-direction convention
  // X: ds1=y, ds2=z; Y: ds1=z, ds2=x; Z: ds1=x, ds2=y.
  int d, side;
  int ds(int which) const {  // dimension of ds1 (which=1) or ds2 (which=2)
    if (d == 0) return which == 1 ? 1 : 2;
    if (d == 1) return which == 1 ? 2 : 0;
    return which == 1 ? 0 : 1;
  }
};

inline int64_t gidx(int b, int x, int y, int z) { return int64_t(b) * BN + cell(x, y, z); }

// taylorSign: parity of the fine cell index along ds (XbaseIndexer etc.)
inline double taylor_sign(const FaceIdx& F, const int c[3], int which) {
  return (c[F.ds(which)] % 2 == 0) ? -1.0 : 1.0;
}
inline bool isBD(const FaceIdx& F, const int c[3], int which) {
  const int v = c[F.ds(which)];
  return v == BS - 1 || v == BS / 2 - 1;
}
inline bool isFD(const FaceIdx& F, const int c[3], int which) {
  const int v = c[F.ds(which)];
  return v == 0 || v == BS / 2;
}
// Nei(info, ix, iy, iz, dist1, dist2)
inline int64_t nei(int b, const FaceIdx& F, const int c[3], int d1, int d2) {
  int q[3] = {c[0], c[1], c[2]};
  q[F.ds(1)] += d1;
  q[F.ds(2)] += d2;
  return gidx(b, q[0], q[1], q[2]);
}

struct Coef {
  int64_t idx;
  double v;
};

// D1 (PoissonSolverExp.h:384-405), scaled by h/4
std::array<Coef, 3> D1(int b, const FaceIdx& F, const int c[3], int which) {
  const int s1 = which == 1, s2 = which == 2;
  auto N = [&](int k) { return nei(b, F, c, s1 * k, s2 * k); };
  const int64_t self = gidx(b, c[0], c[1], c[2]);
  if (isBD(F, c, which)) return {{{N(-2), 1. / 8.}, {N(-1), -1. / 2.}, {self, 3. / 8.}}};
  if (isFD(F, c, which)) return {{{N(2), -1. / 8.}, {N(1), 1. / 2.}, {self, -3. / 8.}}};
  return {{{N(-1), -1. / 8.}, {N(1), 1. / 8.}, {self, 0.}}};
}
// D2 (PoissonSolverExp.h:407-428), scaled by 0.5*(h/4)^2
std::array<Coef, 3> D2(int b, const FaceIdx& F, const int c[3], int which) {
  const int s1 = which == 1, s2 = which == 2;
  auto N = [&](int k) { return nei(b, F, c, s1 * k, s2 * k); };
  const int64_t self = gidx(b, c[0], c[1], c[2]);
  if (isBD(F, c, which)) return {{{N(-2), 1. / 32.}, {N(-1), -1. / 16.}, {self, 1. / 32.}}};
  if (isFD(F, c, which)) return {{{N(2), 1. / 32.}, {N(1), -1. / 16.}, {self, 1. / 32.}}};
  return {{{N(-1), 1. / 32.}, {N(1), 1. / 32.}, {self, -1. / 16.}}};
}
// Dmixed (PoissonSolverExp.h:430-478), scaled by (h/4)^2
std::array<Coef, 4> Dm(int b, const FaceIdx& F, const int c[3]) {
  auto N = [&](int a, int bb) { return nei(b, F, c, a, bb); };
  const bool bd1 = isBD(F, c, 1), bd2 = isBD(F, c, 2), fd1 = isFD(F, c, 1), fd2 = isFD(F, c, 2);
  if (bd1 && bd2)
    return {{{N(0, 0), 1. / 16.}, {N(-1, -1), 1. / 16.}, {N(-1, 0), -1. / 16.}, {N(0, -1), -1. / 16.}}};
  if (fd1 && bd2)
    return {{{N(1, 0), 1. / 16.}, {N(0, -1), 1. / 16.}, {N(1, -1), -1. / 16.}, {N(0, 0), -1. / 16.}}};
  if (bd1 && fd2)
    return {{{N(0, 1), 1. / 16.}, {N(-1, 0), 1. / 16.}, {N(-1, 1), -1. / 16.}, {N(0, 0), -1. / 16.}}};
  if (fd1 && fd2)
    return {{{N(1, 1), 1. / 16.}, {N(0, 0), 1. / 16.}, {N(1, 0), -1. / 16.}, {N(0, 1), -1. / 16.}}};
  if (bd1)
    return {{{N(0, 1), 1. / 32.}, {N(-1, -1), 1. / 32.}, {N(0, -1), -1. / 32.}, {N(-1, 1), -1. / 32.}}};
  if (fd1)
    return {{{N(1, 1), 1. / 32.}, {N(0, -1), 1. / 32.}, {N(1, -1), -1. / 32.}, {N(0, 1), -1. / 32.}}};
  if (bd2)
    return {{{N(1, 0), 1. / 32.}, {N(-1, -1), 1. / 32.}, {N(-1, 0), -1. / 32.}, {N(1, -1), -1. / 32.}}};
  if (fd2)
    return {{{N(1, 1), 1. / 32.}, {N(-1, 0), 1. / 32.}, {N(-1, 1), -1. / 32.}, {N(1, 0), -1. / 32.}}};
  return {{{N(1, 1), 1. / 64.}, {N(-1, -1), 1. / 64.}, {N(1, -1), -1. / 64.}, {N(-1, 1), -1. / 64.}}};
}

// PoissonSolverExp::interpolate (PoissonSolverExp.cpp:112-155)
void interpolate(int bc_, const int cc[3], double hf, int64_t fine_close, int64_t fine_far,
                 double sign, double sds1, double sds2, const FaceIdx& F, Row& row) {
  row[fine_close] += sign * hf * 2. / 3.;
  row[fine_far] += -sign * hf * 1. / 5.;
  const double tf = sign * hf * 8. / 15.;
  row[gidx(bc_, cc[0], cc[1], cc[2])] += tf;
  for (const auto& e : D1(bc_, F, cc, 1)) row[e.idx] += sds1 * tf * e.v;
  for (const auto& e : D1(bc_, F, cc, 2)) row[e.idx] += sds2 * tf * e.v;
  for (const auto& e : D2(bc_, F, cc, 1)) row[e.idx] += tf * e.v;
  for (const auto& e : D2(bc_, F, cc, 2)) row[e.idx] += tf * e.v;
  for (const auto& e : Dm(bc_, F, cc)) row[e.idx] += sds1 * sds2 * tf * e.v;
}

// PoissonSolverExp::makeFlux (PoissonSolverExp.cpp:157-219)
void make_flux(const orc_mesh& m, int b, const int c[3], int d, int side, Row& row) {
  const FaceIdx F{d, side};
  const int f = 2 * d + side;
  const int64_t self = gidx(b, c[0], c[1], c[2]);
  const int k = m.kind[b][f];
  if (k == K_SAME) {
    const int nb_ = m.nbr[b][f][0];
    int q[3] = {c[0], c[1], c[2]};
    q[d] = side ? 0 : BS - 1;  // neiUnif: Xmax of the minus neighbour, Xmin of the plus one
    const double h = m.h[nb_];
    row[gidx(nb_, q[0], q[1], q[2])] += h;
    row[self] += -h;
  } else if (k == K_COARSER) {
    const int bc_ = m.nbr[b][f][0];
    int cc[3];
    for (int e = 0; e < 3; ++e)
      cc[e] = (m.idx[b][e] % 2 == 0) ? (c[e] / 2) : (c[e] / 2 + BS / 2);
    cc[d] = side ? 0 : BS - 1;  // ix_c override of XminIndexer / XmaxIndexer
    int q[3] = {c[0], c[1], c[2]};
    q[d] += side ? -1 : 1;  // neiInward
    const double sds1 = taylor_sign(F, c, 1), sds2 = taylor_sign(F, c, 2);
    const double h = m.h[b];
    interpolate(bc_, cc, h, self, gidx(b, q[0], q[1], q[2]), 1., sds1, sds2, F, row);
    row[self] += -h;
  } else if (k == K_FINER) {
    const int t1 = F.ds(1), t2 = F.ds(2);
    // Zchild: the child touching us; its tangential halves follow our cell index
    const int a1 = c[tan1(d)] >= BS / 2, a2 = c[tan2(d)] >= BS / 2;
    const int ch = m.nbr[b][f][a1 + 2 * a2];
    const double h = m.h[ch];
    // neiFine1..4 with (sign_ds1, sign_ds2) = (-,-), (+,-), (-,+), (+,+)
    for (int q4 = 0; q4 < 4; ++q4) {
      const int e1 = q4 & 1, e2 = q4 >> 1;
      int fc[3], ff[3];
      for (int e = 0; e < 3; ++e) fc[e] = (c[e] % (BS / 2)) * 2;
      fc[t1] += e1;
      fc[t2] += e2;
      fc[d] = side ? 0 : BS - 1;  // Xmin / Xmax of the child, offset 0
      for (int e = 0; e < 3; ++e) ff[e] = fc[e];
      ff[d] = side ? 1 : BS - 2;  // offset 1
      const int64_t close = gidx(ch, fc[0], fc[1], fc[2]);
      const int64_t far = gidx(ch, ff[0], ff[1], ff[2]);
      row[close] += h;
      interpolate(b, c, h, close, far, -1., e1 ? 1. : -1., e2 ? 1. : -1., F, row);
    }
  }
}

// getMat (PoissonSolverExp.cpp:221-373): row `r` of block b
void poisson_row(const orc_mesh& m, int mean_constraint, int b, int x, int y, int z, Row& row) {
  const double h = m.h[b];
  const int64_t self = gidx(b, x, y, z);
  if (mean_constraint == 3 && b == m.mean_block && x == 0 && y == 0 && z == 0) {
    row[self] += h;
    return;
  }
  const int c[3] = {x, y, z};
  for (int d = 0; d < 3; ++d)
    for (int side = 0; side < 2; ++side) {
      const bool valid = side ? c[d] < BS - 1 : c[d] > 0;
      if (valid) {
        int q[3] = {x, y, z};
        q[d] += side ? 1 : -1;
        row[gidx(b, q[0], q[1], q[2])] += h;
        row[self] += -h;
      } else if (m.kind[b][2 * d + side] != K_BOUNDARY) {
        make_flux(m, b, c, d, side, row);
      }
    }
}

}  // namespace

extern "C" int64_t orc_poisson_nnz(orc_mesh* m, int mean_constraint) {
  int64_t nnz = 0;
#pragma omp parallel for reduction(+ : nnz) schedule(dynamic, 4)
  for (int b = 0; b < m->nb; ++b)
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) {
          Row row;
          poisson_row(*m, mean_constraint, b, x, y, z, row);
          nnz += int64_t(row.size());
        }
  return nnz;
}

extern "C" void orc_poisson_csr(orc_mesh* m, int mean_constraint, int64_t* rowptr, int64_t* col,
                                double* val) {
  int64_t p = 0;
  rowptr[0] = 0;
  for (int b = 0; b < m->nb; ++b)
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) {
          Row row;
          poisson_row(*m, mean_constraint, b, x, y, z, row);
          for (const auto& e : row) {
            col[p] = e.first;
            val[p] = e.second;
            ++p;
          }
          rowptr[int64_t(b) * BN + cell(x, y, z) + 1] = p;
        }
}

namespace {
// CSR of the operator, cached inside the mesh per mean_constraint mode.
const orc_mesh::CSR& get_csr(orc_mesh* m, int mc) {
  orc_mesh::CSR* c = &m->csr[mc & 3];
  if (c->rowptr.empty()) {
    const int64_t n = int64_t(m->nb) * BN;
    const int64_t nnz = orc_poisson_nnz(m, mc);
    c->rowptr.resize(n + 1);
    c->col.resize(nnz);
    c->val.resize(nnz);
    orc_poisson_csr(m, mc, c->rowptr.data(), c->col.data(), c->val.data());
  }
  return *c;
}

// A x with the mean constraint of ComputeLHS (PoissonSolverAMR.h:108-172) /
// hd_cusparseSpMV (BiCGSTAB.cu:392-413): mode 1 replaces row (0,0,0) of the
// index-(0,0,0) block by sum(x h^3), mode 2 adds sum(x h^3) h^3 to every row.
void apply_A(orc_mesh* m, int mc, const double* x, double* y) {
  const orc_mesh::CSR& A = get_csr(m, mc);
  const int64_t n = int64_t(m->nb) * BN;
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < n; ++r) {
    double s = 0;
    for (int64_t p = A.rowptr[r]; p < A.rowptr[r + 1]; ++p) s += A.val[p] * x[A.col[p]];
    y[r] = s;
  }
  if (mc == 1 || mc == 2) {
    const double avg = det_sum(m->nb, [&](int64_t b) {
      const double h3 = m->h[b] * m->h[b] * m->h[b];
      double s = 0;
      for (int i = 0; i < BN; ++i) s += x[b * BN + i] * h3;
      return s;
    });
    if (mc == 1) {
      if (m->mean_block >= 0) y[int64_t(m->mean_block) * BN] = avg;
    } else {
#pragma omp parallel for schedule(static)
      for (int b = 0; b < m->nb; ++b) {
        const double h3 = m->h[b] * m->h[b] * m->h[b];
        for (int i = 0; i < BN; ++i) y[int64_t(b) * BN + i] += avg * h3;
      }
    }
  }
}
}  // namespace

extern "C" void orc_poisson_apply(orc_mesh* m, int mean_constraint, const double* x, double* y) {
  apply_A(m, mean_constraint, x, y);
}

// ============================================================================
// Block preconditioners
// ============================================================================

// PoissonSolverExp ctor (PoissonSolverExp.cpp:17-111): P_inv = -(L_D)^-1 for the
// 8^3 Dirichlet 7-point operator L_D (6 on the diagonal, -1 per face neighbour),
// via Cholesky-Crout and a Gauss-Jordan inverse of the factor.
extern "C" void orc_pinv(double* P) {
  const int n = BN;
  auto A = [](int i, int j) -> double {
    if (i == j) return 6.;
    const int ix = i % BS, iy = (i / BS) % BS, iz = i / (BS * BS);
    const int jx = j % BS, jy = (j / BS) % BS, jz = j / (BS * BS);
    return (std::abs(ix - jx) + std::abs(iy - jy) + std::abs(iz - jz)) == 1 ? -1. : 0.;
  };
  std::vector<double> L(size_t(n) * n, 0.0), Li(size_t(n) * n, 0.0);
  for (int i = 0; i < n; ++i) Li[size_t(i) * n + i] = 1.;
  for (int i = 0; i < n; ++i) {
    double s1 = 0;
    for (int k = 0; k < i; ++k) s1 += L[size_t(i) * n + k] * L[size_t(i) * n + k];
    L[size_t(i) * n + i] = std::sqrt(A(i, i) - s1);
    for (int j = i + 1; j < n; ++j) {
      double s2 = 0;
      for (int k = 0; k < i; ++k) s2 += L[size_t(i) * n + k] * L[size_t(j) * n + k];
      L[size_t(j) * n + i] = (A(j, i) - s2) / L[size_t(i) * n + i];
    }
  }
  for (int br = 0; br < n; ++br) {
    const double bsf = 1. / L[size_t(br) * n + br];
    for (int c = 0; c <= br; ++c) Li[size_t(br) * n + c] *= bsf;
    for (int wr = br + 1; wr < n; ++wr) {
      const double wsf = L[size_t(wr) * n + br];
      for (int c = 0; c <= br; ++c) Li[size_t(wr) * n + c] -= wsf * Li[size_t(br) * n + c];
    }
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double aux = 0;
      for (int k = std::max(i, j); k < n; ++k) aux += Li[size_t(k) * n + i] * Li[size_t(k) * n + j];
      P[size_t(i) * n + j] = -aux;
    }
}

// z = (1/h) P_inv p per block (cublasDgemm + blockDscal, BiCGSTAB.cu:526-527)
extern "C" void orc_precond_pinv(orc_mesh* m, const double* P, const double* in, double* out) {
#pragma omp parallel for schedule(static)
  for (int b = 0; b < m->nb; ++b) {
    const double invh = 1.0 / m->h[b];
    const double* pi = in + int64_t(b) * BN;
    double* po = out + int64_t(b) * BN;
    for (int i = 0; i < BN; ++i) {
      double s = 0;
      for (int j = 0; j < BN; ++j) s += P[size_t(i) * BN + j] * pi[j];
      po[i] = invh * s;
    }
  }
}

// Per-block CG on the zero-padded 7-point Laplacian, getZImplParallel and
// kernelPoissonGetZInner (PoissonSolverAMRKernels.cpp:76-80,177-332).
extern "C" void orc_precond_cg(orc_mesh* m, const double* in, double* out) {
  constexpr double kDivEps = 1e-55;
  constexpr double kRel2 = 1e-7 * 1e-7, kAbs2 = 1e-16 * 1e-16;
  constexpr double N = BN;
#pragma omp parallel
  {
    std::vector<double> r(BN), Ax(BN), p(10 * 10 * 10, 0.0);
    auto P = [&](int x, int y, int z) -> double& { return p[(x + 1) + 10 * ((y + 1) + 10 * (z + 1))]; };
#pragma omp for schedule(static)
    for (int b = 0; b < m->nb; ++b) {
      const double invh = 1.0 / m->h[b];
      const double* blk = in + int64_t(b) * BN;
      double* z = out + int64_t(b) * BN;
      double rr = 0;
      for (int zz = 0; zz < BS; ++zz)
        for (int y = 0; y < BS; ++y)
          for (int x = 0; x < BS; ++x) {
            const int i = cell(x, y, zz);
            r[i] = invh * blk[i];
            rr += r[i] * r[i];
            P(x, y, zz) = r[i];
            z[i] = 0;
          }
      const double sqrNorm0 = rr / (N * N);
      if (sqrNorm0 < 1e-32) continue;
      for (int k = 0; k < 100; ++k) {
        double a2 = 0;
        for (int zz = 0; zz < BS; ++zz)
          for (int y = 0; y < BS; ++y)
            for (int x = 0; x < BS; ++x) {
              const int i = cell(x, y, zz);
              Ax[i] = P(x - 1, y, zz) + P(x + 1, y, zz) + P(x, y - 1, zz) + P(x, y + 1, zz) +
                      P(x, y, zz - 1) + P(x, y, zz + 1) - 6 * P(x, y, zz);
              a2 += P(x, y, zz) * Ax[i];
            }
        const double a = rr / (a2 + kDivEps);
        double sqrSum = 0;
        for (int zz = 0; zz < BS; ++zz)
          for (int y = 0; y < BS; ++y)
            for (int x = 0; x < BS; ++x) {
              const int i = cell(x, y, zz);
              z[i] += a * P(x, y, zz);
              r[i] -= a * Ax[i];
              sqrSum += r[i] * r[i];
            }
        const double beta = sqrSum / (rr + kDivEps);
        const double sqrNorm = sqrSum / (N * N);
        if (sqrNorm < kRel2 * sqrNorm0 || sqrNorm < kAbs2) break;
        for (int zz = 0; zz < BS; ++zz)
          for (int y = 0; y < BS; ++y)
            for (int x = 0; x < BS; ++x) P(x, y, zz) = r[cell(x, y, zz)] + beta * P(x, y, zz);
        rr = sqrSum;
      }
      // reset the interior of the padded block for the next block on this thread
      std::fill(p.begin(), p.end(), 0.0);
    }
  }
}

// ============================================================================
// Krylov solvers
// ============================================================================
namespace {
struct Precond {
  orc_mesh* m;
  int kind;  // 0 exact block inverse, 1 block CG
  std::vector<double> P;
  Precond(orc_mesh* mm, int k) : m(mm), kind(k) {
    if (kind == 0) {
      P.resize(size_t(BN) * BN);
      orc_pinv(P.data());
    }
  }
  void apply(const double* in, double* out) {
    if (kind == 0)
      orc_precond_pinv(m, P.data(), in, out);
    else
      orc_precond_cg(m, in, out);
  }
};

double dot(const double* a, const double* b, int64_t n) {
  return det_sum(n, [&](int64_t i) { return a[i] * b[i]; });
}
}  // namespace

// BiCGSTABSolver::main (BiCGSTAB.cu:416-628), one rank.  b and x are modified
// the way getVec does for the mean row (PoissonSolverExp.cpp:402-410).
extern "C" int orc_bicgstab_gpu(orc_mesh* m, int mc, int precond, const double* b_in, double* x,
                                double max_error, double max_rel_error, int max_restarts,
                                int max_iter, double* stats) {
  const int64_t n = int64_t(m->nb) * BN;
  std::vector<double> b(b_in, b_in + n), r(n), rhat(n), p(n), nu(n), t(n), z(n), xopt(n);
  if ((mc == 1 || mc == 3) && m->mean_block >= 0) {
    b[int64_t(m->mean_block) * BN] = 0.;
    x[int64_t(m->mean_block) * BN] = 0.;
  }
  Precond M(m, precond);
  const double eps = 1e-21;
  double alpha = 1, beta = 1, omega = 1, rho_prev = 1, rho_curr = 1;
  apply_A(m, mc, x, nu.data());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - nu[i];
  double error = std::sqrt(dot(r.data(), r.data(), n));
  const double error_init = error;
  double error_opt = error;
  std::copy(x, x + n, xopt.begin());
  rhat = r;
  std::fill(nu.begin(), nu.end(), 0.);
  std::fill(p.begin(), p.end(), 0.);
  int restarts = 0, k = 0;
  bool converged = false;
  for (k = 0; k < max_iter; ++k) {
    rho_curr = dot(rhat.data(), r.data(), n);
    const double nr = dot(r.data(), r.data(), n), nrh = dot(rhat.data(), rhat.data(), n);
    const bool breakdown = rho_curr * rho_curr < 1e-16 * nr * nrh;
    beta = (rho_curr / (rho_prev + eps)) * (alpha / (omega + eps));
    if (breakdown && max_restarts > 0) {
      ++restarts;
      if (restarts >= max_restarts) break;
      rhat = r;
      rho_curr = dot(rhat.data(), rhat.data(), n);
      std::fill(nu.begin(), nu.end(), 0.);
      std::fill(p.begin(), p.end(), 0.);
      rho_prev = 1.;
      alpha = 1.;
      omega = 1.;
      beta = (rho_curr / (rho_prev + eps)) * (alpha / (omega + eps));
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * nu[i]);
    M.apply(p.data(), z.data());
    apply_A(m, mc, z.data(), nu.data());
    alpha = rho_curr / (dot(rhat.data(), nu.data(), n) + eps);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * z[i];
      r[i] -= alpha * nu[i];
    }
    M.apply(r.data(), z.data());
    apply_A(m, mc, z.data(), t.data());
    const double ts = dot(t.data(), r.data(), n), tt = dot(t.data(), t.data(), n);
    omega = ts / (tt + eps);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += omega * z[i];
      r[i] -= omega * t[i];
    }
    error = std::sqrt(dot(r.data(), r.data(), n));
    if (error < error_opt) {
      error_opt = error;
      std::copy(x, x + n, xopt.begin());
      if (error <= max_error || error / error_init <= max_rel_error) {
        converged = true;
        break;
      }
    }
    rho_prev = rho_curr;
  }
  std::copy(xopt.begin(), xopt.end(), x);
  if (stats) {
    stats[0] = k + (converged ? 1 : 0);
    stats[1] = restarts;
    stats[2] = error_init;
    stats[3] = error_opt;
    stats[4] = converged;
  }
  return converged ? 0 : 1;
}

// PoissonSolverAMR::solve (PoissonSolverAMR.cpp:13-358), pipelined BiCGSTAB of
// Cools & Vanroose (Alg. 11) with residual replacement every 50 iterations.
extern "C" int orc_bicgstab_pipelined(orc_mesh* m, int mc, int precond, const double* b_in,
                                      double* x, double max_error, double max_rel_error,
                                      int max_iter, double* stats) {
  const int64_t N = int64_t(m->nb) * BN;
  const double eps = 1e-100;
  const int max_restarts = 100;
  std::vector<double> b(b_in, b_in + N), phat(N), rhat(N), shat(N), what(N), zhat(N), qhat(N),
      s(N), w(N), z(N), t(N), v(N), q(N), r(N), y(N), r0(N), xopt(N);
  if ((mc == 1 || mc > 2) && m->mean_block >= 0) b[int64_t(m->mean_block) * BN] = 0.0;
  r = b;
  Precond M(m, precond);
  apply_A(m, mc, x, r0.data());
#pragma omp parallel for
  for (int64_t i = 0; i < N; ++i) {
    r0[i] = r[i] - r0[i];
    r[i] = r0[i];
  }
  M.apply(r0.data(), rhat.data());
  apply_A(m, mc, rhat.data(), w.data());
  M.apply(w.data(), what.data());
  apply_A(m, mc, what.data(), t.data());
  double alpha = 0, norm = 0, beta = 0, omega = 0, r0r_prev;
  {
    const double t0 = dot(r0.data(), r0.data(), N), t1 = dot(r0.data(), w.data(), N);
    alpha = t0 / (t1 + eps);
    r0r_prev = t0;
    norm = std::sqrt(t0);
  }
  const double init_norm = norm;
  double min_norm = 1e50;
  bool useXopt = false;
  int restarts = 0, k;
  bool converged = false;
  for (k = 0; k < max_iter; ++k) {
    if (k % 50 != 0) {
#pragma omp parallel for
      for (int64_t j = 0; j < N; ++j) {
        phat[j] = rhat[j] + beta * (phat[j] - omega * shat[j]);
        s[j] = w[j] + beta * (s[j] - omega * z[j]);
        shat[j] = what[j] + beta * (shat[j] - omega * zhat[j]);
        z[j] = t[j] + beta * (z[j] - omega * v[j]);
        q[j] = r[j] - alpha * s[j];
        qhat[j] = rhat[j] - alpha * shat[j];
        y[j] = w[j] - alpha * z[j];
      }
    } else {
#pragma omp parallel for
      for (int64_t j = 0; j < N; ++j) phat[j] = rhat[j] + beta * (phat[j] - omega * shat[j]);
      apply_A(m, mc, phat.data(), s.data());
      M.apply(s.data(), shat.data());
      apply_A(m, mc, shat.data(), z.data());
#pragma omp parallel for
      for (int64_t j = 0; j < N; ++j) {
        q[j] = r[j] - alpha * s[j];
        qhat[j] = rhat[j] - alpha * shat[j];
        y[j] = w[j] - alpha * z[j];
      }
    }
    const double qy = dot(q.data(), y.data(), N), yy = dot(y.data(), y.data(), N);
    M.apply(z.data(), zhat.data());
    apply_A(m, mc, zhat.data(), v.data());
    omega = qy / (yy + eps);
    if (k % 50 != 0) {
#pragma omp parallel for
      for (int64_t j = 0; j < N; ++j) {
        x[j] = x[j] + alpha * phat[j] + omega * qhat[j];
        r[j] = q[j] - omega * y[j];
        rhat[j] = qhat[j] - omega * (what[j] - alpha * zhat[j]);
        w[j] = y[j] - omega * (t[j] - alpha * v[j]);
      }
    } else {
#pragma omp parallel for
      for (int64_t j = 0; j < N; ++j) x[j] = x[j] + alpha * phat[j] + omega * qhat[j];
      apply_A(m, mc, x, r.data());
#pragma omp parallel for
      for (int64_t j = 0; j < N; ++j) r[j] = b[j] - r[j];
      M.apply(r.data(), rhat.data());
      apply_A(m, mc, rhat.data(), w.data());
    }
    const double r0r = dot(r0.data(), r.data(), N), r0w = dot(r0.data(), w.data(), N);
    const double r0s = dot(r0.data(), s.data(), N), r0z = dot(r0.data(), z.data(), N);
    const double norm_1 = dot(r.data(), r.data(), N), norm_2 = dot(r0.data(), r0.data(), N);
    norm = norm_1;
    M.apply(w.data(), what.data());
    apply_A(m, mc, what.data(), t.data());
    norm = std::sqrt(norm);
    beta = alpha / (omega + eps) * r0r / (r0r_prev + eps);
    alpha = r0r / (r0w + beta * r0s - beta * omega * r0z);
    double alphat = 1.0 / (omega + eps) + r0w / (r0r + eps) - beta * omega * r0z / (r0r + eps);
    alphat = 1.0 / (alphat + eps);
    if (std::fabs(alphat) < 10 * std::fabs(alpha)) alpha = alphat;
    r0r_prev = r0r;
    const bool serious_breakdown = r0r * r0r < 1e-16 * norm_1 * norm_2;
    if (serious_breakdown && restarts < max_restarts) {
      ++restarts;
      r0 = r;
      M.apply(r0.data(), rhat.data());
      apply_A(m, mc, rhat.data(), w.data());
      const double t0 = dot(r0.data(), r0.data(), N), t1 = dot(r0.data(), w.data(), N);
      M.apply(w.data(), what.data());
      apply_A(m, mc, what.data(), t.data());
      alpha = t0 / (t1 + eps);
      r0r_prev = t0;
      beta = 0.0;
      omega = 0.0;
    }
    if (norm < min_norm) {
      useXopt = true;
      min_norm = norm;
      std::copy(x, x + N, xopt.begin());
    }
    if (norm < max_error || norm / (init_norm + eps) < max_rel_error) {
      converged = true;
      break;
    }
  }
  if (useXopt) std::copy(xopt.begin(), xopt.end(), x);
  if (stats) {
    stats[0] = k + (converged ? 1 : 0);
    stats[1] = restarts;
    stats[2] = init_norm;
    stats[3] = min_norm;
    stats[4] = converged;
  }
  return converged ? 0 : 1;
}

// ============================================================================
// Labs: a block with G ghost layers along the 6 faces (star stencils only).
// Same-level and periodic ghosts copy the neighbour (Cubism BlockLab); boundary
// ghosts follow BlockLabBC::applyBCfaceOpen/Wall (Definitions.h:67-397) for
// vector fields and zero-gradient Neumann for scalar fields.  Coarse-fine
// ghosts (Cubism's interpolation is absent from the reference tree) are our
// definition, shared with the device code:
//   * coarse block, finer neighbour: mean of the 2x2x2 fine cells;
//   * fine block, coarser neighbour C: tensor-product quadratic Lagrange
//     interpolation from C's own cells (normal: C's layers 0,1,2; tangential:
//     3 cells centred on the containing coarse cell, one-sided at C's edges).
// ============================================================================
namespace {

inline void lagrange3(double xi, double w[3]) {
  w[0] = 0.5 * (xi - 1.0) * (xi - 2.0);
  w[1] = -xi * (xi - 2.0);
  w[2] = 0.5 * xi * (xi - 1.0);
}

// Tangential stencil for fine cell t of a fine block whose half is `half`
// inside the coarse block: start node and evaluation point.
inline void tan_stencil(int t, int half, int& n0, double w[3]) {
  const int c = half * (BS / 2) + (t >> 1);
  const double eta = (t & 1) ? 0.25 : -0.25;
  if (c == 0) {
    n0 = 0;
    lagrange3(eta, w);
  } else if (c == BS - 1) {
    n0 = BS - 3;
    lagrange3(2.0 + eta, w);
  } else {
    n0 = c - 1;
    lagrange3(1.0 + eta, w);
  }
}

struct Lab {
  int G, W, ncomp;
  std::vector<double> v;
  Lab(int g, int nc) : G(g), W(BS + 2 * g), ncomp(nc), v(size_t(nc) * W * W * W, 0.0) {}
  double& at(int c, int x, int y, int z) {
    return v[size_t(c) * W * W * W + size_t(z + G) * W * W + size_t(y + G) * W + (x + G)];
  }
};

void fill_lab(const orc_mesh& m, const double* f, int ncomp, int G, int b, bool vector_bc,
              Lab& lab) {
  const int64_t nbn = int64_t(m.nb) * BN;
  auto F = [&](int c, int blk, int x, int y, int z) {
    return f[c * nbn + int64_t(blk) * BN + cell(x, y, z)];
  };
  for (int c = 0; c < ncomp; ++c)
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) lab.at(c, x, y, z) = F(c, b, x, y, z);
  for (int d = 0; d < 3; ++d)
    for (int side = 0; side < 2; ++side) {
      const int f_ = 2 * d + side;
      const int k = m.kind[b][f_];
      const int t1 = tan1(d), t2 = tan2(d);
      for (int l = 1; l <= G; ++l)
        for (int b2 = 0; b2 < BS; ++b2)
          for (int a = 0; a < BS; ++a) {
            int g[3];  // ghost position in lab coordinates of block b
            g[d] = side ? BS - 1 + l : -l;
            g[t1] = a;
            g[t2] = b2;
            for (int c = 0; c < ncomp; ++c) {
              double val = 0;
              if (k == K_SAME) {
                int q[3] = {g[0], g[1], g[2]};
                q[d] = side ? l - 1 : BS - l;
                val = F(c, m.nbr[b][f_][0], q[0], q[1], q[2]);
              } else if (k == K_BOUNDARY) {
                int q[3] = {g[0], g[1], g[2]};
                q[d] = side ? BS - 1 : 0;
                val = F(c, b, q[0], q[1], q[2]);
                if (vector_bc) {
                  const int bc = m.nbr[b][f_][0];
                  if (bc == BC_WALL || c == d) val = -val;
                }
              } else if (k == K_FINER) {
                const int ch = m.nbr[b][f_][(a >> 2) + 2 * (b2 >> 2)];
                double s = 0;
                for (int e2 = 0; e2 < 2; ++e2)
                  for (int e1 = 0; e1 < 2; ++e1)
                    for (int en = 0; en < 2; ++en) {
                      int q[3];
                      const int fl = 2 * (l - 1) + en;  // fine layer from the face
                      q[d] = side ? fl : BS - 1 - fl;
                      q[t1] = 2 * (a & 3) + e1;
                      q[t2] = 2 * (b2 & 3) + e2;
                      s += F(c, ch, q[0], q[1], q[2]);
                    }
                val = 0.125 * s;
              } else {  // K_COARSER
                const int cb = m.nbr[b][f_][0];
                double wn[3], w1[3], w2[3];
                lagrange3((l - 1.5) * 0.5, wn);
                int n1, n2;
                tan_stencil(a, m.idx[b][t1] & 1, n1, w1);
                tan_stencil(b2, m.idx[b][t2] & 1, n2, w2);
                double s = 0;
                for (int i2 = 0; i2 < 3; ++i2)
                  for (int i1 = 0; i1 < 3; ++i1)
                    for (int in = 0; in < 3; ++in) {
                      int q[3];
                      q[d] = side ? in : BS - 1 - in;
                      q[t1] = n1 + i1;
                      q[t2] = n2 + i2;
                      s += wn[in] * w1[i1] * w2[i2] * F(c, cb, q[0], q[1], q[2]);
                    }
                val = s;
              }
              lab.at(c, g[0], g[1], g[2]) = val;
            }
          }
    }
}

// Face value storage for flux correction: per block, per face, ncomp x 64.
struct Faces {
  int nb, ncomp;
  std::vector<double> v;
  Faces(int n, int nc) : nb(n), ncomp(nc), v(size_t(n) * 6 * nc * 64, 0.0) {}
  double& at(int b, int f, int c, int t) { return v[((size_t(b) * 6 + f) * ncomp + c) * 64 + t]; }
};

// Cubism FluxCorrection as used by compute<...>(..., applyFluxCorrection):
// a coarse cell next to a finer face gets its own stored face value (which
// cancels its face term) plus the four fine face values (the fine fluxes).
// comp_mask: which components are corrected on faces normal to d
// (bit c set in comp_mask[d]).
void flux_correct(const orc_mesh& m, Faces& fc, double* out, int ncomp, const int comp_mask[3]) {
  const int64_t nbn = int64_t(m.nb) * BN;
#pragma omp parallel for schedule(dynamic, 4)
  for (int b = 0; b < m.nb; ++b)
    for (int d = 0; d < 3; ++d)
      for (int side = 0; side < 2; ++side) {
        const int f = 2 * d + side;
        if (m.kind[b][f] != K_FINER) continue;
        const int t1 = tan1(d), t2 = tan2(d);
        for (int c2 = 0; c2 < BS; ++c2)
          for (int c1 = 0; c1 < BS; ++c1) {
            const int ch = m.nbr[b][f][(c1 >> 2) + 2 * (c2 >> 2)];
            int q[3];
            q[d] = side ? BS - 1 : 0;
            q[t1] = c1;
            q[t2] = c2;
            for (int c = 0; c < ncomp; ++c) {
              if (!((comp_mask[d] >> c) & 1)) continue;
              double s = fc.at(b, f, c, c1 + BS * c2);
              for (int e2 = 0; e2 < 2; ++e2)
                for (int e1 = 0; e1 < 2; ++e1)
                  s += fc.at(ch, f ^ 1, c, (2 * (c1 & 3) + e1) + BS * (2 * (c2 & 3) + e2));
              out[c * nbn + int64_t(b) * BN + cell(q[0], q[1], q[2])] += s;
            }
          }
      }
}

inline bool has_jump(const orc_mesh& m, int b, int f) {
  return m.kind[b][f] == K_COARSER || m.kind[b][f] == K_FINER;
}

}  // namespace

extern "C" void orc_fill_lab(orc_mesh* m, const double* field, int ncomp, int G, int block,
                             int vector_bc, double* out) {
  Lab lab(G, ncomp);
  fill_lab(*m, field, ncomp, G, block, vector_bc != 0, lab);
  std::memcpy(out, lab.v.data(), lab.v.size() * sizeof(double));
}

// ============================================================================
// Time step control: findMaxU (ProcessHelpers.h:71-94), calcMaxTimestep
// (Simulation.cpp:309-375)
// ============================================================================
extern "C" double orc_max_u(orc_mesh* m, const double* vel, const double* uinf) {
  const int64_t n = int64_t(m->nb) * BN;
  double mx = 0;
#pragma omp parallel for reduction(max : mx) schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double a = std::fabs(vel[i] + uinf[0]);
    const double b = std::fabs(vel[n + i] + uinf[1]);
    const double c = std::fabs(vel[2 * n + i] + uinf[2]);
    mx = std::max(mx, std::max({a, b, c}));
  }
  return mx;
}

extern "C" double orc_dt(double hmin, double nu, double cfl, double umax, int step, int rampup) {
  const double dtDiffusion = (1.0 / 6.0) * hmin * hmin / (nu + (1.0 / 6.0) * hmin * umax);
  const double dtAdvection = hmin / (umax + 1e-8);
  if (step < rampup) {
    const double x = step / (double)rampup;
    const double rampCFL = std::exp(std::log(1e-3) * (1 - x) + std::log(cfl) * x);
    return std::min(dtDiffusion, rampCFL * dtAdvection);
  }
  return std::min(dtDiffusion, cfl * dtAdvection);
}

// ============================================================================
// AdvectionDiffusion (AdvectionDiffusion.cpp:19-322)
// ============================================================================
namespace {

inline double weno5_plus(double um2, double um1, double u, double up1, double up2) {
  const double e = 1e-6;
  const double b1 = 13.0 / 12.0 * std::pow((um2 + u) - 2 * um1, 2) + 0.25 * std::pow((um2 + 3 * u) - 4 * um1, 2);
  const double b2 = 13.0 / 12.0 * std::pow((um1 + up1) - 2 * u, 2) + 0.25 * std::pow(um1 - up1, 2);
  const double b3 = 13.0 / 12.0 * std::pow((u + up2) - 2 * up1, 2) + 0.25 * std::pow((3 * u + up2) - 4 * up1, 2);
  const double g1 = 0.1, g2 = 0.6, g3 = 0.3;
  const double what1 = g1 / std::pow(b1 + e, 2);
  const double what2 = g2 / std::pow(b2 + e, 2);
  const double what3 = g3 / std::pow(b3 + e, 2);
  const double aux = 1.0 / ((what1 + what3) + what2);
  const double w1 = what1 * aux, w2 = what2 * aux, w3 = what3 * aux;
  const double f1 = (11.0 / 6.0) * u + ((1.0 / 3.0) * um2 - (7.0 / 6.0) * um1);
  const double f2 = (5.0 / 6.0) * u + ((-1.0 / 6.0) * um1 + (1.0 / 3.0) * up1);
  const double f3 = (1.0 / 3.0) * u + ((+5.0 / 6.0) * up1 - (1.0 / 6.0) * up2);
  return (w1 * f1 + w3 * f3) + w2 * f2;
}
inline double weno5_minus(double um2, double um1, double u, double up1, double up2) {
  const double e = 1e-6;
  const double b1 = 13.0 / 12.0 * std::pow((um2 + u) - 2 * um1, 2) + 0.25 * std::pow((um2 + 3 * u) - 4 * um1, 2);
  const double b2 = 13.0 / 12.0 * std::pow((um1 + up1) - 2 * u, 2) + 0.25 * std::pow(um1 - up1, 2);
  const double b3 = 13.0 / 12.0 * std::pow((u + up2) - 2 * up1, 2) + 0.25 * std::pow((3 * u + up2) - 4 * up1, 2);
  const double g1 = 0.3, g2 = 0.6, g3 = 0.1;
  const double what1 = g1 / std::pow(b1 + e, 2);
  const double what2 = g2 / std::pow(b2 + e, 2);
  const double what3 = g3 / std::pow(b3 + e, 2);
  const double aux = 1.0 / ((what1 + what3) + what2);
  const double w1 = what1 * aux, w2 = what2 * aux, w3 = what3 * aux;
  const double f1 = (1.0 / 3.0) * u + ((-1.0 / 6.0) * um2 + (5.0 / 6.0) * um1);
  const double f2 = (5.0 / 6.0) * u + ((1.0 / 3.0) * um1 - (1.0 / 6.0) * up1);
  const double f3 = (11.0 / 6.0) * u + ((-7.0 / 6.0) * up1 + (1.0 / 3.0) * up2);
  return (w1 * f1 + w3 * f3) + w2 * f2;
}
inline double deriv(int scheme, double U, double um3, double um2, double um1, double u, double up1,
                    double up2, double up3) {
  if (scheme == 1) {
    double fp, fm;
    if (U > 0) {
      fp = weno5_plus(um2, um1, u, up1, up2);
      fm = weno5_plus(um3, um2, um1, u, up1);
    } else {
      fp = weno5_minus(um1, u, up1, up2, up3);
      fm = weno5_minus(um2, um1, u, up1, up2);
    }
    return fp - fm;
  }
  if (U > 0) return (-2 * um3 + 15 * um2 - 60 * um1 + 20 * u + 30 * up1 - 3 * up2) / 60.;
  return (2 * up3 - 15 * up2 + 60 * up1 - 20 * u - 30 * um1 + 3 * um2) / 60.;
}

void advect_rhs(orc_mesh* m, const double* vel, double* tmpV, double dt, double nu,
                const double* uinf, int scheme, double coef) {
  const int64_t nbn = int64_t(m->nb) * BN;
  Faces fc(m->nb, 3);
#pragma omp parallel
  {
    Lab lab(3, 3);
#pragma omp for schedule(dynamic, 4)
    for (int b = 0; b < m->nb; ++b) {
      fill_lab(*m, vel, 3, 3, b, true, lab);
      const double h = m->h[b], h3 = h * h * h;
      const double facA = -dt / h * h3 * coef;
      const double facD = (nu / h) * (dt / h) * h3 * coef;
      auto L = [&](int c, int x, int y, int z) { return lab.at(c, x, y, z); };
      for (int z = 0; z < BS; ++z)
        for (int y = 0; y < BS; ++y)
          for (int x = 0; x < BS; ++x) {
            const double uA[3] = {L(0, x, y, z) + uinf[0], L(1, x, y, z) + uinf[1], L(2, x, y, z) + uinf[2]};
            double dd[3][3];  // dd[c][dir]
            for (int c = 0; c < 3; ++c) {
              dd[c][0] = deriv(scheme, uA[0], L(c, x - 3, y, z), L(c, x - 2, y, z), L(c, x - 1, y, z), L(c, x, y, z), L(c, x + 1, y, z), L(c, x + 2, y, z), L(c, x + 3, y, z));
              dd[c][1] = deriv(scheme, uA[1], L(c, x, y - 3, z), L(c, x, y - 2, z), L(c, x, y - 1, z), L(c, x, y, z), L(c, x, y + 1, z), L(c, x, y + 2, z), L(c, x, y + 3, z));
              dd[c][2] = deriv(scheme, uA[2], L(c, x, y, z - 3), L(c, x, y, z - 2), L(c, x, y, z - 1), L(c, x, y, z), L(c, x, y, z + 1), L(c, x, y, z + 2), L(c, x, y, z + 3));
            }
            const double duD = ((L(0, x + 1, y, z) + L(0, x - 1, y, z)) + ((L(0, x, y + 1, z) + L(0, x, y - 1, z)) + (L(0, x, y, z + 1) + L(0, x, y, z - 1)))) - 6 * L(0, x, y, z);
            const double dvD = ((L(1, x, y + 1, z) + L(1, x, y - 1, z)) + ((L(1, x, y, z + 1) + L(1, x, y, z - 1)) + (L(1, x + 1, y, z) + L(1, x - 1, y, z)))) - 6 * L(1, x, y, z);
            const double dwD = ((L(2, x, y, z + 1) + L(2, x, y, z - 1)) + ((L(2, x + 1, y, z) + L(2, x - 1, y, z)) + (L(2, x, y + 1, z) + L(2, x, y - 1, z)))) - 6 * L(2, x, y, z);
            const double duA = uA[0] * dd[0][0] + (uA[1] * dd[0][1] + uA[2] * dd[0][2]);
            const double dvA = uA[1] * dd[1][1] + (uA[2] * dd[1][2] + uA[0] * dd[1][0]);
            const double dwA = uA[2] * dd[2][2] + (uA[0] * dd[2][0] + uA[1] * dd[2][1]);
            const int64_t o = int64_t(b) * BN + cell(x, y, z);
            tmpV[o] += facA * duA + facD * duD;
            tmpV[nbn + o] += facA * dvA + facD * dvD;
            tmpV[2 * nbn + o] += facA * dwA + facD * dwD;
          }
      // face fluxes (AdvectionDiffusion.cpp:138-213)
      for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) {
          const int f = 2 * d + side;
          if (!has_jump(*m, b, f)) continue;
          const int t1 = tan1(d), t2 = tan2(d);
          for (int b2 = 0; b2 < BS; ++b2)
            for (int a = 0; a < BS; ++a) {
              int q[3], g[3];
              q[d] = side ? BS - 1 : 0;
              q[t1] = a;
              q[t2] = b2;
              for (int e = 0; e < 3; ++e) g[e] = q[e];
              g[d] += side ? 1 : -1;
              for (int c = 0; c < 3; ++c)
                fc.at(b, f, c, a + BS * b2) = facD * (L(c, q[0], q[1], q[2]) - L(c, g[0], g[1], g[2]));
            }
        }
    }
  }
  const int mask[3] = {7, 7, 7};
  flux_correct(*m, fc, tmpV, 3, mask);
}

}  // namespace

extern "C" void orc_advect_rhs(orc_mesh* m, const double* vel, double* tmpV, double dt, double nu,
                               const double* uinf, int scheme, double coef) {
  advect_rhs(m, vel, tmpV, dt, nu, uinf, scheme, coef);
}

extern "C" void orc_advect_diffuse(orc_mesh* m, double* vel, double* tmpV, double dt, double nu,
                                   const double* uinf, int scheme) {
  const int64_t nbn = int64_t(m->nb) * BN;
  const double alpha[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
  const double beta[3] = {-5.0 / 9.0, -153.0 / 128.0, 0.0};
  std::fill(tmpV, tmpV + 3 * nbn, 0.0);
  for (int s = 0; s < 3; ++s) {
    advect_rhs(m, vel, tmpV, dt, nu, uinf, scheme, 1.0);
#pragma omp parallel for schedule(static)
    for (int b = 0; b < m->nb; ++b) {
      const double ih3 = alpha[s] / (m->h[b] * m->h[b] * m->h[b]);
      for (int c = 0; c < 3; ++c)
        for (int i = 0; i < BN; ++i) {
          const int64_t o = c * nbn + int64_t(b) * BN + i;
          vel[o] += tmpV[o] * ih3;
          tmpV[o] *= beta[s];
        }
    }
  }
}

// ============================================================================
// Penalization (Penalization.cpp:18-109)
// ============================================================================
extern "C" void orc_penalize(orc_mesh* m, double* vel, const double* chi, const int32_t* slot,
                             int nslots, const double* chi_o, const double* udef_o,
                             const double* ob, double dt, double lambda, int implicit,
                             double* force_out) {
  const int64_t nbn = int64_t(m->nb) * BN;
  const double lambdaFac = implicit ? lambda : 1.0 / dt;
  double F[6] = {0, 0, 0, 0, 0, 0};
  std::vector<std::array<double, 6>> per(m->nb, {0, 0, 0, 0, 0, 0});
#pragma omp parallel for schedule(dynamic, 4)
  for (int b = 0; b < m->nb; ++b) {
    const int s = slot[b];
    if (s < 0) continue;
    const double h = m->h[b], dv = h * h * h;
    const double org[3] = {m->idx[b][0] * BS * h, m->idx[b][1] * BS * h, m->idx[b][2] * BS * h};
    double FX = 0, FY = 0, FZ = 0, TX = 0, TY = 0, TZ = 0;
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) {
          const int i = cell(x, y, z);
          const double CHI = chi_o[size_t(s) * BN + i];
          if (chi[int64_t(b) * BN + i] > CHI) continue;
          if (CHI <= 0) continue;
          double p[3] = {org[0] + (x + 0.5) * h, org[1] + (y + 0.5) * h, org[2] + (z + 0.5) * h};
          p[0] -= ob[0];
          p[1] -= ob[1];
          p[2] -= ob[2];
          const double* vv = ob + 3;
          const double* om = ob + 6;
          const double U[3] = {
              vv[0] + om[1] * p[2] - om[2] * p[1] + udef_o[(0 * size_t(nslots) + s) * BN + i],
              vv[1] + om[2] * p[0] - om[0] * p[2] + udef_o[(1 * size_t(nslots) + s) * BN + i],
              vv[2] + om[0] * p[1] - om[1] * p[0] + udef_o[(2 * size_t(nslots) + s) * BN + i]};
          const double X = implicit ? (CHI > 0.5 ? 1.0 : 0.0) : CHI;
          const double penalFac = implicit ? X * lambdaFac / (1 + X * lambdaFac * dt) : X * lambdaFac;
          const int64_t o = int64_t(b) * BN + i;
          const double FPX = penalFac * (U[0] - vel[o]);
          const double FPY = penalFac * (U[1] - vel[nbn + o]);
          const double FPZ = penalFac * (U[2] - vel[2 * nbn + o]);
          vel[o] = vel[o] + dt * FPX;
          vel[nbn + o] = vel[nbn + o] + dt * FPY;
          vel[2 * nbn + o] = vel[2 * nbn + o] + dt * FPZ;
          FX += dv * FPX;
          FY += dv * FPY;
          FZ += dv * FPZ;
          TX += dv * (p[1] * FPZ - p[2] * FPY);
          TY += dv * (p[2] * FPX - p[0] * FPZ);
          TZ += dv * (p[0] * FPY - p[1] * FPX);
        }
    per[b] = {FX, FY, FZ, TX, TY, TZ};
  }
  for (int b = 0; b < m->nb; ++b)
    for (int q = 0; q < 6; ++q) F[q] += per[b][q];
  if (force_out)
    for (int q = 0; q < 6; ++q) force_out[q] = F[q];
}

// ============================================================================
// PressureProjection (PressureProjection.cpp:16-468)
// ============================================================================
namespace {

// tmpV = udef where grid chi <= obstacle chi (kernelUpdateTmpV, :202-242)
void udef_to_tmpV(orc_mesh* m, const double* chi, const int32_t* slot, int nslots,
                  const double* chi_o, const double* udef_o, double* tmpV) {
  const int64_t nbn = int64_t(m->nb) * BN;
  std::fill(tmpV, tmpV + 3 * nbn, 0.0);
  if (!slot) return;
#pragma omp parallel for schedule(static)
  for (int b = 0; b < m->nb; ++b) {
    const int s = slot[b];
    if (s < 0) continue;
    for (int i = 0; i < BN; ++i) {
      if (chi[int64_t(b) * BN + i] > chi_o[size_t(s) * BN + i]) continue;
      for (int c = 0; c < 3; ++c)
        tmpV[c * nbn + int64_t(b) * BN + i] += udef_o[(c * size_t(nslots) + s) * BN + i];
    }
  }
}

// KernelPressureRHS (:96-199) with flux correction
void pressure_rhs(orc_mesh* m, const double* vel, const double* tmpV, const double* chi, double dt,
                  double* lhs) {
  Faces fc(m->nb, 1);
#pragma omp parallel
  {
    Lab lab(1, 3), ulab(1, 3);
#pragma omp for schedule(dynamic, 4)
    for (int b = 0; b < m->nb; ++b) {
      fill_lab(*m, vel, 3, 1, b, true, lab);
      fill_lab(*m, tmpV, 3, 1, b, true, ulab);
      const double h = m->h[b], fac = 0.5 * h * h / dt;
      for (int z = 0; z < BS; ++z)
        for (int y = 0; y < BS; ++y)
          for (int x = 0; x < BS; ++x) {
            const int64_t o = int64_t(b) * BN + cell(x, y, z);
            double p = fac * (lab.at(0, x + 1, y, z) - lab.at(0, x - 1, y, z) + lab.at(1, x, y + 1, z) -
                              lab.at(1, x, y - 1, z) + lab.at(2, x, y, z + 1) - lab.at(2, x, y, z - 1));
            const double divUs = ulab.at(0, x + 1, y, z) - ulab.at(0, x - 1, y, z) + ulab.at(1, x, y + 1, z) -
                                 ulab.at(1, x, y - 1, z) + ulab.at(2, x, y, z + 1) - ulab.at(2, x, y, z - 1);
            p += -chi[o] * fac * divUs;
            lhs[o] = p;
          }
      for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) {
          const int f = 2 * d + side;
          if (!has_jump(*m, b, f)) continue;
          const int t1 = tan1(d), t2 = tan2(d);
          for (int b2 = 0; b2 < BS; ++b2)
            for (int a = 0; a < BS; ++a) {
              int q[3], g[3];
              q[d] = side ? BS - 1 : 0;
              q[t1] = a;
              q[t2] = b2;
              for (int e = 0; e < 3; ++e) g[e] = q[e];
              g[d] += side ? 1 : -1;
              const double c = chi[int64_t(b) * BN + cell(q[0], q[1], q[2])];
              const double sg = side ? -1.0 : 1.0;
              fc.at(b, f, 0, a + BS * b2) =
                  sg * fac * (lab.at(d, g[0], g[1], g[2]) + lab.at(d, q[0], q[1], q[2])) -
                  sg * c * fac * (ulab.at(d, g[0], g[1], g[2]) + ulab.at(d, q[0], q[1], q[2]));
            }
        }
    }
  }
  const int mask[3] = {1, 1, 1};
  flux_correct(*m, fc, lhs, 1, mask);
}

// KernelDivPressure (:16-94): out = h * Lap7(p) with flux correction
void div_pressure(orc_mesh* m, const double* p, double* out) {
  Faces fc(m->nb, 1);
#pragma omp parallel
  {
    Lab lab(1, 1);
#pragma omp for schedule(dynamic, 4)
    for (int b = 0; b < m->nb; ++b) {
      fill_lab(*m, p, 1, 1, b, false, lab);
      const double fac = m->h[b];
      for (int z = 0; z < BS; ++z)
        for (int y = 0; y < BS; ++y)
          for (int x = 0; x < BS; ++x)
            out[int64_t(b) * BN + cell(x, y, z)] =
                fac * (lab.at(0, x + 1, y, z) + lab.at(0, x - 1, y, z) + lab.at(0, x, y + 1, z) +
                       lab.at(0, x, y - 1, z) + lab.at(0, x, y, z + 1) + lab.at(0, x, y, z - 1) -
                       6.0 * lab.at(0, x, y, z));
      for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) {
          const int f = 2 * d + side;
          if (!has_jump(*m, b, f)) continue;
          const int t1 = tan1(d), t2 = tan2(d);
          for (int b2 = 0; b2 < BS; ++b2)
            for (int a = 0; a < BS; ++a) {
              int q[3], g[3];
              q[d] = side ? BS - 1 : 0;
              q[t1] = a;
              q[t2] = b2;
              for (int e = 0; e < 3; ++e) g[e] = q[e];
              g[d] += side ? 1 : -1;
              fc.at(b, f, 0, a + BS * b2) = fac * (lab.at(0, q[0], q[1], q[2]) - lab.at(0, g[0], g[1], g[2]));
            }
        }
    }
  }
  const int mask[3] = {1, 1, 1};
  flux_correct(*m, fc, out, 1, mask);
}

// KernelGradP (:244-323) + velocity update (:451-467)
void grad_update(orc_mesh* m, double* vel, const double* p, double dt) {
  const int64_t nbn = int64_t(m->nb) * BN;
  std::vector<double> g(3 * nbn);
  Faces fc(m->nb, 3);
#pragma omp parallel
  {
    Lab lab(1, 1);
#pragma omp for schedule(dynamic, 4)
    for (int b = 0; b < m->nb; ++b) {
      fill_lab(*m, p, 1, 1, b, false, lab);
      const double h = m->h[b], fac = -0.5 * dt * h * h;
      for (int z = 0; z < BS; ++z)
        for (int y = 0; y < BS; ++y)
          for (int x = 0; x < BS; ++x) {
            const int64_t o = int64_t(b) * BN + cell(x, y, z);
            g[o] = fac * (lab.at(0, x + 1, y, z) - lab.at(0, x - 1, y, z));
            g[nbn + o] = fac * (lab.at(0, x, y + 1, z) - lab.at(0, x, y - 1, z));
            g[2 * nbn + o] = fac * (lab.at(0, x, y, z + 1) - lab.at(0, x, y, z - 1));
          }
      for (int d = 0; d < 3; ++d)
        for (int side = 0; side < 2; ++side) {
          const int f = 2 * d + side;
          if (!has_jump(*m, b, f)) continue;
          const int t1 = tan1(d), t2 = tan2(d);
          for (int b2 = 0; b2 < BS; ++b2)
            for (int a = 0; a < BS; ++a) {
              int q[3], gg[3];
              q[d] = side ? BS - 1 : 0;
              q[t1] = a;
              q[t2] = b2;
              for (int e = 0; e < 3; ++e) gg[e] = q[e];
              gg[d] += side ? 1 : -1;
              const double sg = side ? -1.0 : 1.0;
              fc.at(b, f, d, a + BS * b2) = sg * fac * (lab.at(0, gg[0], gg[1], gg[2]) + lab.at(0, q[0], q[1], q[2]));
            }
        }
    }
  }
  const int mask[3] = {1, 2, 4};
  flux_correct(*m, fc, g.data(), 3, mask);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < m->nb; ++b) {
    const double fac = 1.0 / (m->h[b] * m->h[b] * m->h[b]);
    for (int c = 0; c < 3; ++c)
      for (int i = 0; i < BN; ++i) {
        const int64_t o = c * nbn + int64_t(b) * BN + i;
        vel[o] += fac * g[o];
      }
  }
}

}  // namespace

extern "C" void orc_pressure_rhs(orc_mesh* m, const double* vel, const double* pres,
                                 const double* chi, const int32_t* slot, int nslots,
                                 const double* chi_o, const double* udef_o, double dt, int step,
                                 double* lhs) {
  const int64_t nbn = int64_t(m->nb) * BN;
  std::vector<double> tmpV(3 * nbn);
  std::vector<double> zchi;
  if (!chi) {
    zchi.assign(nbn, 0.0);
    chi = zchi.data();
  }
  udef_to_tmpV(m, chi, slot, nslots, chi_o, udef_o, tmpV.data());
  pressure_rhs(m, vel, tmpV.data(), chi, dt, lhs);
  if (step > 2) {
    std::vector<double> dp(nbn);
    div_pressure(m, pres, dp.data());
    for (int64_t i = 0; i < nbn; ++i) lhs[i] -= dp[i];
  }
}

extern "C" void orc_grad_update(orc_mesh* m, double* vel, const double* pres, double dt) {
  grad_update(m, vel, pres, dt);
}

// ComputeDissipation's KernelDissipation (ComputeDissipation.cpp:17-109): the
// 20 volume integrals of the diagnostics file from one-layer labs of the
// velocity and the pressure, cell by cell in block order; positions relative
// to the domain centre (extents / 2).
extern "C" void orc_dissipation(orc_mesh* m, const double* vel, const double* pres, const double* chi, double nu,
                                double* out) {
  double Q[20] = {0};
  const double center[3] = {0.5 * m->bpd[0] * BS * m->h0, 0.5 * m->bpd[1] * BS * m->h0,
                            0.5 * m->bpd[2] * BS * m->h0};
  Lab L(1, 3), P(1, 1);
  for (int b = 0; b < m->nb; ++b) {
    fill_lab(*m, vel, 3, 1, b, true, L);
    fill_lab(*m, pres, 1, 1, b, false, P);
    const double h = m->h[b];
    const double hCube = std::pow(h, 3), inv2h = .5 / h, invHh = 1 / (h * h);
    for (int iz = 0; iz < BS; ++iz)
      for (int iy = 0; iy < BS; ++iy)
        for (int ix = 0; ix < BS; ++ix) {
          auto U = [&](int c, int dx, int dy, int dz) { return L.at(c, ix + dx, iy + dy, iz + dz); };
          const double X = chi ? chi[int64_t(b) * BN + cell(ix, iy, iz)] : 0.0;
          const double PX = (m->idx[b][0] * BS + ix + 0.5) * h - center[0];
          const double PY = (m->idx[b][1] * BS + iy + 0.5) * h - center[1];
          const double PZ = (m->idx[b][2] * BS + iz + 0.5) * h - center[2];
          const double WX = inv2h * ((U(2, 0, 1, 0) - U(2, 0, -1, 0)) - (U(1, 0, 0, 1) - U(1, 0, 0, -1)));
          const double WY = inv2h * ((U(0, 0, 0, 1) - U(0, 0, 0, -1)) - (U(2, 1, 0, 0) - U(2, -1, 0, 0)));
          const double WZ = inv2h * ((U(1, 1, 0, 0) - U(1, -1, 0, 0)) - (U(0, 0, 1, 0) - U(0, 0, -1, 0)));
          const double dPdx = inv2h * (P.at(0, ix + 1, iy, iz) - P.at(0, ix - 1, iy, iz));
          const double dPdy = inv2h * (P.at(0, ix, iy + 1, iz) - P.at(0, ix, iy - 1, iz));
          const double dPdz = inv2h * (P.at(0, ix, iy, iz + 1) - P.at(0, ix, iy, iz - 1));
          double lap[3];
          for (int c = 0; c < 3; ++c)
            lap[c] = invHh * (U(c, 1, 0, 0) + U(c, -1, 0, 0) + U(c, 0, 1, 0) + U(c, 0, -1, 0) + U(c, 0, 0, 1) +
                              U(c, 0, 0, -1) - 6 * U(c, 0, 0, 0));
          const double u0 = U(0, 0, 0, 0), u1 = U(1, 0, 0, 0), u2 = U(2, 0, 0, 0);
          const double V1 = lap[0] * u0 + lap[1] * u1 + lap[2] * u2;
          const double D11 = inv2h * (U(0, 1, 0, 0) - U(0, -1, 0, 0));
          const double D22 = inv2h * (U(1, 0, 1, 0) - U(1, 0, -1, 0));
          const double D33 = inv2h * (U(2, 0, 0, 1) - U(2, 0, 0, -1));
          const double D12 = inv2h * (U(0, 0, 1, 0) - U(0, 0, -1, 0) + U(1, 1, 0, 0) - U(1, -1, 0, 0)) / 2;
          const double D13 = inv2h * (U(0, 0, 0, 1) - U(0, 0, 0, -1) + U(2, 1, 0, 0) - U(2, -1, 0, 0)) / 2;
          const double D23 = inv2h * (U(2, 0, 1, 0) - U(2, 0, -1, 0) + U(1, 0, 0, 1) - U(1, 0, 0, -1)) / 2;
          const double V2 = D11 * D11 + D22 * D22 + D33 * D33 + 2 * (D12 * D12 + D13 * D13 + D23 * D23);
          Q[0] += hCube * WX;
          Q[1] += hCube * WY;
          Q[2] += hCube * WZ;
          Q[3] += hCube / 2 * (PY * WZ - PZ * WY);
          Q[4] += hCube / 2 * (PZ * WX - PX * WZ);
          Q[5] += hCube / 2 * (PX * WY - PY * WX);
          Q[6] += hCube * u0;
          Q[7] += hCube * u1;
          Q[8] += hCube * u2;
          Q[9] += hCube / 3 * (PX * (PY * WY + PZ * WZ) - WX * (PY * PY + PZ * PZ));
          Q[10] += hCube / 3 * (PY * (PX * WX + PZ * WZ) - WY * (PX * PX + PZ * PZ));
          Q[11] += hCube / 3 * (PZ * (PX * WX + PY * WY) - WZ * (PX * PX + PY * PY));
          Q[12] += hCube * (PY * u2 - PZ * u1);
          Q[13] += hCube * (PZ * u0 - PX * u2);
          Q[14] += hCube * (PX * u1 - PY * u0);
          Q[15] -= (1 - X) * hCube * (dPdx * u0 + dPdy * u1 + dPdz * u2);
          Q[16] += (1 - X) * hCube * nu * (V1 + 2 * V2);
          Q[17] += hCube * (WX * u0 + WY * u1 + WZ * u2);
          Q[18] += hCube * (u0 * u0 + u1 * u1 + u2 * u2) / 2;
          Q[19] += hCube * std::sqrt(WX * WX + WY * WY + WZ * WZ);
        }
  }
  for (int i = 0; i < 20; ++i) out[i] = Q[i];
}

extern "C" void orc_pressure_project(orc_mesh* m, double* vel, double* pres, const double* chi,
                                     const int32_t* slot, int nslots, const double* chi_o,
                                     const double* udef_o, double dt, int step, int mc, int solver,
                                     double tol, double tol_rel, double* stats, double* lhs_out) {
  const int64_t nbn = int64_t(m->nb) * BN;
  std::vector<double> pOld(pres, pres + nbn), lhs(nbn);
  orc_pressure_rhs(m, vel, pres, chi, slot, nslots, chi_o, udef_o, dt, step, lhs.data());
  std::fill(pres, pres + nbn, 0.0);  // initial guess 0 (:381-393)
  if (lhs_out) std::copy(lhs.begin(), lhs.end(), lhs_out);
  if (solver == 0)
    orc_bicgstab_gpu(m, mc, 0, lhs.data(), pres, tol, tol_rel, 100, 1000, stats);
  else
    orc_bicgstab_pipelined(m, mc, 1, lhs.data(), pres, tol, tol_rel, 1000, stats);
  // zero mean (:404-431) and incremental pressure (:435-446)
  double avg = det_sum(m->nb, [&](int64_t b) {
    const double vv = m->h[b] * m->h[b] * m->h[b];
    double s = 0;
    for (int i = 0; i < BN; ++i) s += pres[b * BN + i] * vv;
    return s;
  });
  const double avg1 = det_sum(m->nb, [&](int64_t b) {
    const double vv = m->h[b] * m->h[b] * m->h[b];
    double s = 0;
    for (int i = 0; i < BN; ++i) s += vv;
    return s;
  });
  avg = avg / avg1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nbn; ++i) pres[i] -= avg;
  if (step > 2)
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nbn; ++i) pres[i] += pOld[i];
  grad_update(m, vel, pres, dt);
}

// ============================================================================
// Learned preconditioner network (no reference counterpart; written from the
// definition of a 3-D convolution).  Parameters in one array, in this order:
// W0[co][tap] (1 -> C, 'valid' on the 10^3 input), b0[C], W1[co][ci][tap],
// b1[C], W2[co][ci][tap], b2[C], W3[ci][tap] (C -> 1), b3; tap = kx + 3 ky + 9 kz.
// The layers are linear (no activation) and the bias slots are not used, so
// the network is a linear map of its input (it serves as a preconditioner);
// layers 1-3 are zero-padded 'same' convolutions on the 8^3 block.  Loss:
// mean over samples and cells of (z - target)^2; the bias gradients are 0.
// ============================================================================
namespace {
struct CnnDims {
  int C, oW0, oB0, oW1, oB1, oW2, oB2, oW3, oB3, n;
  explicit CnnDims(int c) : C(c) {
    oW0 = 0;
    oB0 = oW0 + C * 27;
    oW1 = oB0 + C;
    oB1 = oW1 + C * C * 27;
    oW2 = oB1 + C;
    oB2 = oW2 + C * C * 27;
    oW3 = oB2 + C;
    oB3 = oW3 + C * 27;
    n = oB3 + 1;
  }
};
inline bool inb(int x, int y, int z) { return x >= 0 && y >= 0 && z >= 0 && x < BS && y < BS && z < BS; }
}  // namespace

extern "C" int orc_cnn_nparam(int C) { return CnnDims(C).n; }

extern "C" void orc_cnn_fwd_grad(int nblk, int C, const double* P, const float* in, const float* target,
                                 float* out, double* grad, double* loss) {
  const CnnDims D(C);
  const double scale = 1.0 / (double(nblk) * BN);
  std::vector<double> G(grad ? D.n : 0, 0.0);
  double L = 0;
#pragma omp parallel
  {
    std::vector<double> a1(C * BN), a2(C * BN), a3(C * BN), z(BN), d3(C * BN), d2(C * BN), d1(C * BN);
    std::vector<double> g(grad ? D.n : 0, 0.0);
    double l = 0;
#pragma omp for schedule(static)
    for (int n = 0; n < nblk; ++n) {
      const float* x = in + size_t(n) * 1000;
      auto X = [&](int xx, int yy, int zz) { return double(x[xx + 10 * (yy + 10 * zz)]); };
      for (int co = 0; co < C; ++co)
        for (int c = 0; c < BN; ++c) {
          const int xx = c % 8, yy = (c / 8) % 8, zz = c / 64;
          double s = 0.0;
          for (int t = 0; t < 27; ++t) s += P[D.oW0 + co * 27 + t] * X(xx + t % 3, yy + (t / 3) % 3, zz + t / 9);
          a1[co * BN + c] = s;
        }
      auto same = [&](const std::vector<double>& a, int oW, std::vector<double>& o) {
        for (int co = 0; co < C; ++co)
          for (int c = 0; c < BN; ++c) {
            const int xx = c % 8, yy = (c / 8) % 8, zz = c / 64;
            double s = 0.0;
            for (int ci = 0; ci < C; ++ci)
              for (int t = 0; t < 27; ++t) {
                const int X2 = xx + t % 3 - 1, Y2 = yy + (t / 3) % 3 - 1, Z2 = zz + t / 9 - 1;
                if (inb(X2, Y2, Z2)) s += P[oW + (co * C + ci) * 27 + t] * a[ci * BN + cell(X2, Y2, Z2)];
              }
            o[co * BN + c] = s;
          }
      };
      same(a1, D.oW1, a2);
      same(a2, D.oW2, a3);
      for (int c = 0; c < BN; ++c) {
        const int xx = c % 8, yy = (c / 8) % 8, zz = c / 64;
        double s = 0.0;
        for (int ci = 0; ci < C; ++ci)
          for (int t = 0; t < 27; ++t) {
            const int X2 = xx + t % 3 - 1, Y2 = yy + (t / 3) % 3 - 1, Z2 = zz + t / 9 - 1;
            if (inb(X2, Y2, Z2)) s += P[D.oW3 + ci * 27 + t] * a3[ci * BN + cell(X2, Y2, Z2)];
          }
        z[c] = s;
        if (out) out[size_t(n) * BN + c] = float(s);
      }
      if (!target) continue;
      for (int c = 0; c < BN; ++c) {
        const double e = z[c] - target[size_t(n) * BN + c];
        l += e * e;
        z[c] = 2.0 * e * scale;  // dL/dz
      }
      if (!grad) continue;
      // layer 3
      for (int c = 0; c < BN; ++c) {
        const int xx = c % 8, yy = (c / 8) % 8, zz = c / 64;
        for (int ci = 0; ci < C; ++ci)
          for (int t = 0; t < 27; ++t) {
            const int X2 = xx + t % 3 - 1, Y2 = yy + (t / 3) % 3 - 1, Z2 = zz + t / 9 - 1;
            if (inb(X2, Y2, Z2)) g[D.oW3 + ci * 27 + t] += a3[ci * BN + cell(X2, Y2, Z2)] * z[c];
          }
      }
      std::fill(d3.begin(), d3.end(), 0.0);
      for (int c = 0; c < BN; ++c) {
        const int xx = c % 8, yy = (c / 8) % 8, zz = c / 64;
        for (int ci = 0; ci < C; ++ci)
          for (int t = 0; t < 27; ++t) {
            const int X2 = xx + t % 3 - 1, Y2 = yy + (t / 3) % 3 - 1, Z2 = zz + t / 9 - 1;
            if (inb(X2, Y2, Z2)) d3[ci * BN + cell(X2, Y2, Z2)] += P[D.oW3 + ci * 27 + t] * z[c];
          }
      }
      auto back_same = [&](const std::vector<double>& a, const std::vector<double>& dp, int oW,
                           std::vector<double>* da) {
        for (int co = 0; co < C; ++co)
          for (int c = 0; c < BN; ++c) {
            const double dv = dp[co * BN + c];
            if (dv == 0) continue;
            const int xx = c % 8, yy = (c / 8) % 8, zz = c / 64;
            for (int ci = 0; ci < C; ++ci)
              for (int t = 0; t < 27; ++t) {
                const int X2 = xx + t % 3 - 1, Y2 = yy + (t / 3) % 3 - 1, Z2 = zz + t / 9 - 1;
                if (!inb(X2, Y2, Z2)) continue;
                const int cc = cell(X2, Y2, Z2);
                g[oW + (co * C + ci) * 27 + t] += a[ci * BN + cc] * dv;
                if (da) (*da)[ci * BN + cc] += P[oW + (co * C + ci) * 27 + t] * dv;
              }
          }
      };
      std::fill(d2.begin(), d2.end(), 0.0);
      back_same(a2, d3, D.oW2, &d2);
      std::fill(d1.begin(), d1.end(), 0.0);
      back_same(a1, d2, D.oW1, &d1);
      for (int co = 0; co < C; ++co)
        for (int c = 0; c < BN; ++c) {
          const double dv = d1[co * BN + c];
          if (dv == 0) continue;
          const int xx = c % 8, yy = (c / 8) % 8, zz = c / 64;
          for (int t = 0; t < 27; ++t) g[D.oW0 + co * 27 + t] += X(xx + t % 3, yy + (t / 3) % 3, zz + t / 9) * dv;
        }
    }
#pragma omp critical(orc_cnn)
    {
      L += l;
      for (size_t i = 0; i < g.size(); ++i) G[i] += g[i];
    }
  }
  if (grad)
    for (int i = 0; i < D.n; ++i) grad[i] = G[i];
  if (loss) *loss = L * scale;
}

// ============================================================================
// Obstacle creation (CreateObstacles, ObstaclesCreate.cpp:18-148): for every
// block the body's box touches (Obstacle::create_base, Obstacle.h:139-160,
// isTouching of Sphere.cpp:31-45 / Ellipsoid.cpp:266-280, margin (2+SURFDH)
// sim.hmin with SURFDH = 1, ObstacleBlock.h:16), the signed distance on the
// block and a one-cell halo (FillBlocksBase, ObstacleLibrary.h:44-59), then
// chi by Towers' FDMH eq. (14) with the chi moments
// (KernelCharacteristicFunction, ObstaclesCreate.cpp:28-88), the grid chi
// max(chi, grid chi) and the centre of mass (kernelComputeGridCoM, :128-148).
// Block origins are index * 8 * h and cell centres origin + (i + 0.5) h
// (Cubism's BlockInfo::pos; Cubism is not in the reference tree).
// ============================================================================
namespace obst_orc {

constexpr double EPS = std::numeric_limits<double>::epsilon();
constexpr int IMAX = 2 * std::numeric_limits<double>::max_exponent;

// Ellipsoid.cpp:22-69 (distPointEllipseSpecial): e0 >= e1, y in the first quadrant.
double ellipse_special(const double e[2], const double y[2], double x[2]) {
  if (y[1] > 0) {
    if (y[0] > 0) {
      const double esqr[2] = {e[0] * e[0], e[1] * e[1]};
      const double ey[2] = {e[0] * y[0], e[1] * y[1]};
      double t0 = -esqr[1] + ey[1];
      double t1 = -esqr[1] + std::sqrt(ey[0] * ey[0] + ey[1] * ey[1]);
      double t = t0;
      for (int i = 0; i < IMAX; ++i) {
        t = 0.5 * (t0 + t1);
        if (std::fabs(t - t0) < EPS || std::fabs(t - t1) < EPS) break;
        const double r[2] = {ey[0] / (t + esqr[0]), ey[1] / (t + esqr[1])};
        const double f = r[0] * r[0] + r[1] * r[1] - 1;
        if (f > 0) t0 = t;
        else if (f < 0) t1 = t;
        else break;
      }
      x[0] = esqr[0] * y[0] / (t + esqr[0]);
      x[1] = esqr[1] * y[1] / (t + esqr[1]);
      const double d[2] = {x[0] - y[0], x[1] - y[1]};
      return std::sqrt(d[0] * d[0] + d[1] * d[1]);
    }
    x[0] = 0;
    x[1] = e[1];
    return std::fabs(y[1] - e[1]);
  }
  const double denom0 = e[0] * e[0] - e[1] * e[1];
  const double e0y0 = e[0] * y[0];
  if (e0y0 < denom0) {
    const double x0de0 = e0y0 / denom0;
    const double x0de0sqr = x0de0 * x0de0;
    x[0] = e[0] * x0de0;
    x[1] = e[1] * std::sqrt(std::fabs(1.0 - x0de0sqr));
    const double d0 = x[0] - y[0];
    return std::sqrt(d0 * d0 + x[1] * x[1]);
  }
  x[0] = e[0];
  x[1] = 0;
  return std::fabs(y[0] - e[0]);
}

// Ellipsoid.cpp:117-203 (distPointEllipsoidSpecial): e0 >= e1 >= e2, first octant.
double ellipsoid_special(const double e[3], const double y[3], double x[3]) {
  if (y[2] > 0) {
    if (y[1] > 0) {
      if (y[0] > 0) {
        const double esq[3] = {e[0] * e[0], e[1] * e[1], e[2] * e[2]};
        const double ey[3] = {e[0] * y[0], e[1] * y[1], e[2] * y[2]};
        double t0 = -esq[2] + ey[2];
        double t1 = -esq[2] + std::sqrt(ey[0] * ey[0] + ey[1] * ey[1] + ey[2] * ey[2]);
        double t = t0;
        for (int i = 0; i < IMAX; ++i) {
          t = 0.5 * (t0 + t1);
          if (std::fabs(t - t0) < EPS || std::fabs(t - t1) < EPS) break;
          const double r[3] = {ey[0] / (t + esq[0]), ey[1] / (t + esq[1]), ey[2] / (t + esq[2])};
          const double f = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] - 1;
          if (f > 0) t0 = t;
          else if (f < 0) t1 = t;
          else break;
        }
        x[0] = esq[0] * y[0] / (t + esq[0]);
        x[1] = esq[1] * y[1] / (t + esq[1]);
        x[2] = esq[2] * y[2] / (t + esq[2]);
        const double d[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
        return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      }
      x[0] = 0;
      const double et[2] = {e[1], e[2]}, yt[2] = {y[1], y[2]};
      double xt[2];
      const double dist = ellipse_special(et, yt, xt);
      x[1] = xt[0];
      x[2] = xt[1];
      return dist;
    }
    x[1] = 0;
    if (y[0] > 0) {
      const double et[2] = {e[0], e[2]}, yt[2] = {y[0], y[2]};
      double xt[2];
      const double dist = ellipse_special(et, yt, xt);
      x[0] = xt[0];
      x[2] = xt[1];
      return dist;
    }
    x[0] = 0;
    x[2] = e[2];
    return std::fabs(y[2] - e[2]);
  }
  const double denom[2] = {e[0] * e[0] - e[2] * e[2], e[1] * e[1] - e[2] * e[2]};
  const double ey[2] = {e[0] * y[0], e[1] * y[1]};
  if (ey[0] < denom[0] && ey[1] < denom[1]) {
    const double xde[2] = {ey[0] / denom[0], ey[1] / denom[1]};
    const double xdesqr[2] = {xde[0] * xde[0], xde[1] * xde[1]};
    const double discr = 1 - xdesqr[0] - xdesqr[1];
    if (discr > 0) {
      x[0] = e[0] * xde[0];
      x[1] = e[1] * xde[1];
      x[2] = e[2] * std::sqrt(discr);
      const double d[2] = {x[0] - y[0], x[1] - y[1]};
      return std::sqrt(d[0] * d[0] + d[1] * d[1] + x[2] * x[2]);
    }
    x[2] = 0;
    return ellipse_special(e, y, x);
  }
  x[2] = 0;
  return ellipse_special(e, y, x);
}

// Ellipsoid.cpp:211-258 (distancePointEllipsoid): reflection and axis order.
double ellipsoid_distance(const double e[3], const double y[3], double x[3]) {
  const bool reflect[3] = {y[0] < 0, y[1] < 0, y[2] < 0};
  int permute[3];
  if (e[0] < e[1]) {
    if (e[2] < e[0]) { permute[0] = 1; permute[1] = 0; permute[2] = 2; }
    else if (e[2] < e[1]) { permute[0] = 1; permute[1] = 2; permute[2] = 0; }
    else { permute[0] = 2; permute[1] = 1; permute[2] = 0; }
  } else {
    if (e[2] < e[1]) { permute[0] = 0; permute[1] = 1; permute[2] = 2; }
    else if (e[2] < e[0]) { permute[0] = 0; permute[1] = 2; permute[2] = 1; }
    else { permute[0] = 2; permute[1] = 0; permute[2] = 1; }
  }
  int invpermute[3];
  for (int i = 0; i < 3; ++i) invpermute[permute[i]] = i;
  double locE[3], locY[3], locX[3];
  for (int i = 0; i < 3; ++i) {
    const int j = permute[i];
    locE[i] = e[j];
    locY[i] = y[j];
    if (reflect[j]) locY[i] = -locY[i];
  }
  const double distance = ellipsoid_special(locE, locY, locX);
  for (int i = 0; i < 3; ++i) {
    const int j = invpermute[i];
    if (reflect[j]) locX[j] = -locX[j];
    x[i] = locX[j];
  }
  return distance;
}

struct Body {
  int kind;  // 0 sphere, 1 ellipsoid
  double pos[3], radius, e[3], R[3][3], box[3][2];
  // Sphere.cpp:47-51; Ellipsoid.cpp:282-299 with positive inside (the
  // obstacle contract, ObstacleLibrary.h:30-32)
  double sdf(double xo, double yo, double zo) const {
    if (kind == 0) {
      const double dx = xo - pos[0], dy = yo - pos[1], dz = zo - pos[2];
      return radius - std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    const double p[3] = {xo - pos[0], yo - pos[1], zo - pos[2]};
    const double t[3] = {R[0][0] * p[0] + R[0][1] * p[1] + R[0][2] * p[2],
                         R[1][0] * p[0] + R[1][1] * p[1] + R[1][2] * p[2],
                         R[2][0] * p[0] + R[2][1] * p[1] + R[2][2] * p[2]};
    double xs[3];
    const double dist = ellipsoid_distance(e, t, xs);
    const double Dcentre = t[0] * t[0] + t[1] * t[1] + t[2] * t[2];
    const double Dsurf = xs[0] * xs[0] + xs[1] * xs[1] + xs[2] * xs[2];
    return Dcentre > Dsurf ? -dist : dist;
  }
  bool touching(const double minp[3], const double maxp[3]) const {
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
      const double lo = std::max(minp[d], box[d][0]), hi = std::min(maxp[d], box[d][1]);
      ok = ok && hi - lo > 0;
    }
    return ok;
  }
};

}  // namespace obst_orc

// The body of orc_create_obstacle's arguments (fill box with the reference's
// safety margin of 3 finest cells; rotation from the quaternion).
static obst_orc::Body orc_make_body(const orc_mesh* m, int kind, const double* centre, const double* shape,
                                    const double* q) {
  using namespace obst_orc;
  Body B{};
  B.kind = kind;
  for (int d = 0; d < 3; ++d) B.pos[d] = centre[d];
  const double h = m->hmin, safety = (2 + 1) * h;
  if (kind == 0) {
    B.radius = shape[0];
    for (int d = 0; d < 3; ++d) {
      B.box[d][0] = B.pos[d] - (B.radius + safety);
      B.box[d][1] = B.pos[d] + (B.radius + safety);
    }
  } else {
    for (int d = 0; d < 3; ++d) B.e[d] = shape[d];
    const double maxAxis = std::max({B.e[0], B.e[1], B.e[2]});
    for (int d = 0; d < 3; ++d) {
      B.box[d][0] = B.pos[d] - 2 * (maxAxis + safety);
      B.box[d][1] = B.pos[d] + 2 * (maxAxis + safety);
    }
    const double w = q[0], x = q[1], y = q[2], z = q[3];
    const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y + z * w), 2 * (x * z - y * w)},
                            {2 * (x * y - z * w), 1 - 2 * (x * x + z * z), 2 * (y * z + x * w)},
                            {2 * (x * z + y * w), 2 * (y * z - x * w), 1 - 2 * (x * x + y * y)}};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B.R[i][j] = R[i][j];
  }
  return B;
}

extern "C" int orc_create_obstacle(orc_mesh* m, int kind, const double* centre, const double* shape,
                                   const double* q, int32_t* obst_slot, int32_t* block_of_slot, double* chi_o,
                                   double* chi_grid, double* mom) {
  using namespace obst_orc;
  const Body B = orc_make_body(m, kind, centre, shape, q);
  const int nb = m->nb;
  std::fill(chi_grid, chi_grid + size_t(nb) * BN, 0.0);
  int ns = 0;
  std::vector<double> bm(4 * size_t(nb), 0.0);  // per-block CoM_x, CoM_y, CoM_z, mass
  for (int b = 0; b < nb; ++b) {
    obst_slot[b] = -1;
    const double hb = m->h[b];
    double org[3], minp[3], maxp[3];
    for (int d = 0; d < 3; ++d) {
      org[d] = m->idx[b][d] * 8 * hb;
      minp[d] = org[d] + hb * (0 + 0.5);
      maxp[d] = org[d] + hb * (BS - 1 + 0.5);
    }
    if (!B.touching(minp, maxp)) continue;
    const int s = ns++;
    obst_slot[b] = s;
    block_of_slot[s] = b;
    static thread_local double lab[BS + 2][BS + 2][BS + 2];
    for (int iz = -1; iz < BS + 1; ++iz)
      for (int iy = -1; iy < BS + 1; ++iy)
        for (int ix = -1; ix < BS + 1; ++ix)
          lab[iz + 1][iy + 1][ix + 1] =
              B.sdf(org[0] + hb * (ix + 0.5), org[1] + hb * (iy + 0.5), org[2] + hb * (iz + 0.5));
    const double inv2h = .5 / hb, vol = hb * hb * hb;
    double* CHI = chi_o + size_t(s) * BN;
    double* M4 = &bm[4 * size_t(b)];
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) {
          const double s0 = lab[z + 1][y + 1][x + 1];
          double chi;
          if (s0 > +hb || s0 < -hb) {
            chi = s0 > 0 ? 1 : 0;
          } else {
            const double distPx = lab[z + 1][y + 1][x + 2], distMx = lab[z + 1][y + 1][x];
            const double distPy = lab[z + 1][y + 2][x + 1], distMy = lab[z + 1][y][x + 1];
            const double distPz = lab[z + 2][y + 1][x + 1], distMz = lab[z][y + 1][x + 1];
            const double gradUX = inv2h * (distPx - distMx);
            const double gradUY = inv2h * (distPy - distMy);
            const double gradUZ = inv2h * (distPz - distMz);
            const double gradUSq = gradUX * gradUX + gradUY * gradUY + gradUZ * gradUZ + EPS;
            const double gradIX = inv2h * (std::max(0.0, distPx) - std::max(0.0, distMx));
            const double gradIY = inv2h * (std::max(0.0, distPy) - std::max(0.0, distMy));
            const double gradIZ = inv2h * (std::max(0.0, distPz) - std::max(0.0, distMz));
            const double numH = gradIX * gradUX + gradIY * gradUY + gradIZ * gradUZ;
            chi = numH / gradUSq;
          }
          const int c = x + BS * y + BS * BS * z;
          CHI[c] = chi;
          chi_grid[size_t(b) * BN + c] = std::max(chi, chi_grid[size_t(b) * BN + c]);
          const double p[3] = {org[0] + hb * (x + 0.5), org[1] + hb * (y + 0.5), org[2] + hb * (z + 0.5)};
          M4[0] += chi * vol * p[0];
          M4[1] += chi * vol * p[1];
          M4[2] += chi * vol * p[2];
          M4[3] += chi * vol;
        }
  }
  // kernelComputeGridCoM: block sums in block order
  for (int k = 0; k < 4; ++k) mom[k] = 0.0;
  for (int b = 0; b < nb; ++b)
    if (obst_slot[b] >= 0)
      for (int k = 0; k < 4; ++k) mom[k] += bm[4 * size_t(b) + k];
  return ns;
}

// ============================================================================
// Surface forces (ComputeForces, FluidSolidForces.cpp:14-229).  Surface
// points of each obstacle block (the second loop of
// KernelCharacteristicFunction, ObstaclesCreate.cpp:83-117, and
// ObstacleBlock::write): nrm[3][ns][512] = -Delta grad(sdf) where the block's
// chi gradient is not zero and Delta > epsilon, else 0.
// ============================================================================
extern "C" void orc_obstacle_surface(orc_mesh* m, int kind, const double* centre, const double* shape,
                                     const double* q, int ns, const int32_t* block_of_slot, const double* chi_o,
                                     double* nrm) {
  using namespace obst_orc;
  const Body B = orc_make_body(m, kind, centre, shape, q);
  for (int sl = 0; sl < ns; ++sl) {
    const int b = block_of_slot[sl];
    const double hb = m->h[b];
    double org[3];
    for (int d = 0; d < 3; ++d) org[d] = m->idx[b][d] * 8 * hb;
    double lab[BS + 2][BS + 2][BS + 2];
    for (int iz = -1; iz < BS + 1; ++iz)
      for (int iy = -1; iy < BS + 1; ++iy)
        for (int ix = -1; ix < BS + 1; ++ix)
          lab[iz + 1][iy + 1][ix + 1] =
              B.sdf(org[0] + hb * (ix + 0.5), org[1] + hb * (iy + 0.5), org[2] + hb * (iz + 0.5));
    const double* CHI = chi_o + size_t(sl) * BN;
    auto C = [&](int x, int y, int z) { return CHI[x + BS * y + BS * BS * z]; };
    const double inv2h = .5 / hb, fac1 = .5 * hb * hb;
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) {
          const double gradUX = inv2h * (lab[z + 1][y + 1][x + 2] - lab[z + 1][y + 1][x]);
          const double gradUY = inv2h * (lab[z + 1][y + 2][x + 1] - lab[z + 1][y][x + 1]);
          const double gradUZ = inv2h * (lab[z + 2][y + 1][x + 1] - lab[z][y + 1][x + 1]);
          const double gradUSq = gradUX * gradUX + gradUY * gradUY + gradUZ * gradUZ + EPS;
          const double gradHX = x == 0 ? 2.0 * (-0.5 * C(x + 2, y, z) + 2.0 * C(x + 1, y, z) - 1.5 * C(x, y, z))
                                : (x == BS - 1 ? 2.0 * (1.5 * C(x, y, z) - 2.0 * C(x - 1, y, z) + 0.5 * C(x - 2, y, z))
                                               : (C(x + 1, y, z) - C(x - 1, y, z)));
          const double gradHY = y == 0 ? 2.0 * (-0.5 * C(x, y + 2, z) + 2.0 * C(x, y + 1, z) - 1.5 * C(x, y, z))
                                : (y == BS - 1 ? 2.0 * (1.5 * C(x, y, z) - 2.0 * C(x, y - 1, z) + 0.5 * C(x, y - 2, z))
                                               : (C(x, y + 1, z) - C(x, y - 1, z)));
          const double gradHZ = z == 0 ? 2.0 * (-0.5 * C(x, y, z + 2) + 2.0 * C(x, y, z + 1) - 1.5 * C(x, y, z))
                                : (z == BS - 1 ? 2.0 * (1.5 * C(x, y, z) - 2.0 * C(x, y, z - 1) + 0.5 * C(x, y, z - 2))
                                               : (C(x, y, z + 1) - C(x, y, z - 1)));
          const int c = x + BS * y + BS * BS * z;
          double n3[3] = {0, 0, 0};
          if (!(gradHX * gradHX + gradHY * gradHY + gradHZ * gradHZ < 1e-12)) {
            const double numD = gradHX * gradUX + gradHY * gradUY + gradHZ * gradUZ;
            const double Delta = fac1 * numD / gradUSq;
            if (Delta > EPS) {
              n3[0] = -Delta * gradUX;
              n3[1] = -Delta * gradUY;
              n3[2] = -Delta * gradUZ;
            }
          }
          for (int d = 0; d < 3; ++d) nrm[(size_t(d) * ns + sl) * BN + c] = n3[d];
        }
  }
}

// KernelComputeForces::visit over the slots (vel [3][n], udef [3][ns][512],
// kin = centre of mass, translation and angular velocity); the lab is read
// at the block's own level (periodic wrap; cells of no block at that level
// are NaN).  qoi[19]: surface force, pressure force, viscous force, torque
// (3 each), drag, thrust, Pout, PoutBnd, defPower, defPowerBnd, pLocom.
// Returns the surface points whose result is not finite.
extern "C" int orc_compute_forces(orc_mesh* m, const double* vel, const double* pres, const double* chi_grid, int ns,
                                  const int32_t* block_of_slot, const double* nrm, const double* udef, double nu,
                                  const double* kin, double* qoi) {
  const size_t n = size_t(m->nb) * BN;
  const double* CM = kin;
  const double* uT = kin + 3;
  const double* om = kin + 6;
  double velUnit[3] = {0, 0, 0};
  const double vn = std::sqrt(uT[0] * uT[0] + uT[1] * uT[1] + uT[2] * uT[2]);
  if (vn > 1e-9)
    for (int d = 0; d < 3; ++d) velUnit[d] = uT[d] / vn;
  for (int k = 0; k < 19; ++k) qoi[k] = 0.0;
  int bad = 0;
  const double c0 = -137. / 60., c1 = 5., c2 = -5., c3 = 10. / 3., c4 = -5. / 4., c5 = 1. / 5.;
  auto inrange = [](int i) { return i >= -4 && i < BS + 4; };
  for (int sl = 0; sl < ns; ++sl) {
    const int b = block_of_slot[sl], L = m->level[b];
    const double h = m->h[b], _1oH = nu / h;
    // field value at cell (x, y, z) of the block's frame, at its level
    auto val = [&](const double* f, int x, int y, int z) {
      int g[3] = {m->idx[b][0] * BS + x, m->idx[b][1] * BS + y, m->idx[b][2] * BS + z};
      int bi[3];
      for (int d = 0; d < 3; ++d) {
        const int N = (m->bpd[d] << L) * BS;
        if (g[d] < 0 || g[d] >= N) {
          if (m->bc[d] != BC_PERIODIC) return std::numeric_limits<double>::quiet_NaN();
          g[d] = ((g[d] % N) + N) % N;
        }
        bi[d] = g[d] / BS;
      }
      const int nbk = m->find(L, bi[0], bi[1], bi[2]);
      if (nbk < 0) return std::numeric_limits<double>::quiet_NaN();
      return f[size_t(nbk) * BN + (g[0] - bi[0] * BS) + BS * (g[1] - bi[1] * BS) + BS * BS * (g[2] - bi[2] * BS)];
    };
    for (int t = 0; t < BN; ++t) {
      const double normX = nrm[(0 * size_t(ns) + sl) * BN + t], normY = nrm[(1 * size_t(ns) + sl) * BN + t],
                   normZ = nrm[(2 * size_t(ns) + sl) * BN + t];
      if (normX == 0.0 && normY == 0.0 && normZ == 0.0) continue;
      const int ix = t % BS, iy = (t / BS) % BS, iz = t / (BS * BS);
      const double p[3] = {m->idx[b][0] * 8 * h + h * (ix + 0.5), m->idx[b][1] * 8 * h + h * (iy + 0.5),
                           m->idx[b][2] * 8 * h + h * (iz + 0.5)};
      const double norm = 1.0 / std::sqrt(normX * normX + normY * normY + normZ * normZ);
      const double dx = normX * norm, dy = normY * norm, dz = normZ * norm;
      int x = ix, y = iy, z = iz;
      for (int kk = 0; kk < 5; ++kk) {
        const int dxi = int(std::round(kk * dx)), dyi = int(std::round(kk * dy)), dzi = int(std::round(kk * dz));
        if (ix + dxi + 1 >= BS + 4 || ix + dxi - 1 < -4) continue;
        if (iy + dyi + 1 >= BS + 4 || iy + dyi - 1 < -4) continue;
        if (iz + dzi + 1 >= BS + 4 || iz + dzi - 1 < -4) continue;
        x = ix + dxi;
        y = iy + dyi;
        z = iz + dzi;
        if (val(chi_grid, x, y, z) < 0.01) break;
      }
      const int sx = normX > 0 ? +1 : -1, sy = normY > 0 ? +1 : -1, sz = normZ > 0 ? +1 : -1;
      double G[3][3];
      for (int c = 0; c < 3; ++c) {
        const double* f = vel + c * n;
        auto l = [&](int X, int Y, int Z) { return val(f, X, Y, Z); };
        double dveldx, dveldy, dveldz;
        if (inrange(x + 5 * sx))
          dveldx = sx * (c0 * l(x, y, z) + c1 * l(x + sx, y, z) + c2 * l(x + 2 * sx, y, z) + c3 * l(x + 3 * sx, y, z) +
                         c4 * l(x + 4 * sx, y, z) + c5 * l(x + 5 * sx, y, z));
        else if (inrange(x + 2 * sx))
          dveldx = sx * (-1.5 * l(x, y, z) + 2.0 * l(x + sx, y, z) - 0.5 * l(x + 2 * sx, y, z));
        else
          dveldx = sx * (l(x + sx, y, z) - l(x, y, z));
        if (inrange(y + 5 * sy))
          dveldy = sy * (c0 * l(x, y, z) + c1 * l(x, y + sy, z) + c2 * l(x, y + 2 * sy, z) + c3 * l(x, y + 3 * sy, z) +
                         c4 * l(x, y + 4 * sy, z) + c5 * l(x, y + 5 * sy, z));
        else if (inrange(y + 2 * sy))
          dveldy = sy * (-1.5 * l(x, y, z) + 2.0 * l(x, y + sy, z) - 0.5 * l(x, y + 2 * sy, z));
        else
          dveldy = sx * (l(x, y + sy, z) - l(x, y, z));
        if (inrange(z + 5 * sz))
          dveldz = sz * (c0 * l(x, y, z) + c1 * l(x, y, z + sz) + c2 * l(x, y, z + 2 * sz) + c3 * l(x, y, z + 3 * sz) +
                         c4 * l(x, y, z + 4 * sz) + c5 * l(x, y, z + 5 * sz));
        else if (inrange(z + 2 * sz))
          dveldz = sz * (-1.5 * l(x, y, z) + 2.0 * l(x, y, z + sz) - 0.5 * l(x, y, z + 2 * sz));
        else
          dveldz = sz * (l(x, y, z + sz) - l(x, y, z));
        const double dveldx2 = l(x - 1, y, z) - 2.0 * l(x, y, z) + l(x + 1, y, z);
        const double dveldy2 = l(x, y - 1, z) - 2.0 * l(x, y, z) + l(x, y + 1, z);
        const double dveldz2 = l(x, y, z - 1) - 2.0 * l(x, y, z) + l(x, y, z + 1);
        double dxy, dyz, dxz;
        if (inrange(x + 2 * sx) && inrange(y + 2 * sy))
          dxy = sx * sy * (-0.5 * (-1.5 * l(x + 2 * sx, y, z) + 2 * l(x + 2 * sx, y + sy, z) - 0.5 * l(x + 2 * sx, y + 2 * sy, z)) +
                           2 * (-1.5 * l(x + sx, y, z) + 2 * l(x + sx, y + sy, z) - 0.5 * l(x + sx, y + 2 * sy, z)) -
                           1.5 * (-1.5 * l(x, y, z) + 2 * l(x, y + sy, z) - 0.5 * l(x, y + 2 * sy, z)));
        else
          dxy = sx * sy * (l(x + sx, y + sy, z) - l(x + sx, y, z)) - (l(x, y + sy, z) - l(x, y, z));
        if (inrange(y + 2 * sy) && inrange(z + 2 * sz))
          dyz = sy * sz * (-0.5 * (-1.5 * l(x, y + 2 * sy, z) + 2 * l(x, y + 2 * sy, z + sz) - 0.5 * l(x, y + 2 * sy, z + 2 * sz)) +
                           2 * (-1.5 * l(x, y + sy, z) + 2 * l(x, y + sy, z + sz) - 0.5 * l(x, y + sy, z + 2 * sz)) -
                           1.5 * (-1.5 * l(x, y, z) + 2 * l(x, y, z + sz) - 0.5 * l(x, y, z + 2 * sz)));
        else
          dyz = sy * sz * (l(x, y + sy, z + sz) - l(x, y + sy, z)) - (l(x, y, z + sz) - l(x, y, z));
        if (inrange(x + 2 * sx) && inrange(z + 2 * sz))
          dxz = sx * sz * (-0.5 * (-1.5 * l(x, y, z + 2 * sz) + 2 * l(x + sx, y, z + 2 * sz) - 0.5 * l(x + 2 * sx, y, z + 2 * sz)) +
                           2 * (-1.5 * l(x, y, z + sz) + 2 * l(x + sx, y, z + sz) - 0.5 * l(x + 2 * sx, y, z + sz)) -
                           1.5 * (-1.5 * l(x, y, z) + 2 * l(x + sx, y, z) - 0.5 * l(x + 2 * sx, y, z)));
        else
          dxz = sx * sz * (l(x + sx, y, z + sz) - l(x, y, z + sz)) - (l(x + sx, y, z) - l(x, y, z));
        G[c][0] = dveldx + dveldx2 * (ix - x) + dxy * (iy - y) + dxz * (iz - z);
        G[c][1] = dveldy + dveldy2 * (iy - y) + dyz * (iz - z) + dxy * (ix - x);
        G[c][2] = dveldz + dveldz2 * (iz - z) + dxz * (ix - x) + dyz * (iy - y);
      }
      const double P = pres[size_t(b) * BN + t];
      const double fXV = _1oH * (G[0][0] * normX + G[0][1] * normY + G[0][2] * normZ);
      const double fYV = _1oH * (G[1][0] * normX + G[1][1] * normY + G[1][2] * normZ);
      const double fZV = _1oH * (G[2][0] * normX + G[2][1] * normY + G[2][2] * normZ);
      const double fXP = -P * normX, fYP = -P * normY, fZP = -P * normZ;
      const double fXT = fXV + fXP, fYT = fYV + fYP, fZT = fZV + fZP;
      const double vX = vel[0 * n + size_t(b) * BN + t], vY = vel[1 * n + size_t(b) * BN + t],
                   vZ = vel[2 * n + size_t(b) * BN + t];
      const size_t us = size_t(ns) * BN, ud = size_t(sl) * BN + t;
      const double forcePar = fXT * velUnit[0] + fYT * velUnit[1] + fZT * velUnit[2];
      const double powOut = fXT * vX + fYT * vY + fZT * vZ;
      const double powDef = fXT * udef[ud] + fYT * udef[us + ud] + fZT * udef[2 * us + ud];
      const double r[3] = {p[0] - CM[0], p[1] - CM[1], p[2] - CM[2]};
      const double uS[3] = {uT[0] + om[1] * r[2] - r[1] * om[2], uT[1] + om[2] * r[0] - r[2] * om[0],
                            uT[2] + om[0] * r[1] - r[0] * om[1]};
      const double v[19] = {fXT, fYT, fZT, fXP, fYP, fZP, fXV, fYV, fZV,
                            r[1] * fZT - r[2] * fYT, r[2] * fXT - r[0] * fZT, r[0] * fYT - r[1] * fXT,
                            -.5 * (forcePar - std::fabs(forcePar)), .5 * (forcePar + std::fabs(forcePar)), powOut,
                            std::min(0.0, powOut), powDef, std::min(0.0, powDef),
                            fXT * uS[0] + fYT * uS[1] + fZT * uS[2]};
      bool finite = true;
      for (int k = 0; k < 19; ++k) finite = finite && std::isfinite(v[k]);
      if (!finite) {
        ++bad;
        continue;
      }
      for (int k = 0; k < 19; ++k) qoi[k] += v[k];
    }
  }
  return bad;
}

// ============================================================================
// Mesh adaptation (Simulation::adaptMesh, Simulation.cpp:128-149).  The
// vorticity of KernelVorticity (ProcessHelpers.h:96-118, scaled by 1/h^3 as
// ComputeVorticity does, :219-234) and GradChiOnTmp's marks (:17-69) give a
// per-block indicator; the refine / compress / transfer rules stand in for
// Cubism's MeshAdaptation, which is not in the reference tree (the same rules
// as the library's, written here independently):
//   indicator: max over cells of |omega| (cells with clamped chi > 0.9: 0;
//     on level levelMaxVorticity-1 < levelMax-1: values >= Rtol count as
//     (Rtol+Ctol)/2); 1e10 if 1e-5 < clamped chi < 0.9 anywhere in the block
//     or its face ghost layers (2 layers on the finest level, else 1);
//   refine at >= Rtol below levelMax-1, then 2:1 balance over 26 neighbours;
//   merge eight sibling leaves all < Ctol unless a leaf finer than them
//   touches the parent; transfer: copy / parent + central slopes at +-1/4 /
//   mean of the eight children.
// ============================================================================
extern "C" void orc_adapt_indicator(orc_mesh* m, const double* vel, const double* chi, int level_max,
                                    int level_max_vort, double rtol, double ctol, double* out) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int b = 0; b < m->nb; ++b) {
    Lab u(1, 3), c(2, 1);
    fill_lab(*m, vel, 3, 1, b, true, u);
    fill_lab(*m, chi, 1, 2, b, false, c);
    const int lev = m->level[b];
    const int offset = lev == level_max - 1 ? 2 : 1;
    auto clamp01 = [](double s) { return std::max(std::min(s, 1.0), 0.0); };
    bool iface = false;
    for (int z = -offset; z < BS + offset; ++z)
      for (int y = -offset; y < BS + offset; ++y)
        for (int x = -offset; x < BS + offset; ++x) {
          const int out_of = (x < 0 || x >= BS) + (y < 0 || y >= BS) + (z < 0 || z >= BS);
          if (out_of > 1) continue;  // face ghost layers only
          const double s = clamp01(c.at(0, x, y, z));
          if (s > 0.00001 && s < 0.9) iface = true;
        }
    const double h = m->h[b], inv2h = .5 * h * h, fac = 1.0 / (h * h * h);
    const bool clamp_vort = lev == level_max_vort - 1 && level_max_vort < level_max;
    double vmax = 0.0;
    for (int z = 0; z < BS; ++z)
      for (int y = 0; y < BS; ++y)
        for (int x = 0; x < BS; ++x) {
          double w[3] = {inv2h * ((u.at(2, x, y + 1, z) - u.at(2, x, y - 1, z)) -
                                  (u.at(1, x, y, z + 1) - u.at(1, x, y, z - 1))),
                         inv2h * ((u.at(0, x, y, z + 1) - u.at(0, x, y, z - 1)) -
                                  (u.at(2, x + 1, y, z) - u.at(2, x - 1, y, z))),
                         inv2h * ((u.at(1, x + 1, y, z) - u.at(1, x - 1, y, z)) -
                                  (u.at(0, x, y + 1, z) - u.at(0, x, y - 1, z)))};
          for (double& v : w) v *= fac;
          double mag = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
          if (clamp_vort && mag >= rtol) {
            w[0] = 0.5 * (rtol + ctol);
            w[1] = w[2] = 0.0;
            mag = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
          }
          if (clamp01(c.at(0, x, y, z)) > 0.9) mag = 0.0;
          vmax = std::max(vmax, mag);
        }
    out[b] = iface ? 1e10 : vmax;
  }
}

namespace adapt_orc {
using Key = std::array<int, 4>;
struct Leaves {
  const orc_mesh* m;
  std::set<Key> s;
  // the leaf containing level-l position p (at level <= l), or level -1
  Key cover(int l, int i, int j, int k) const {
    for (int a = l; a >= 0; --a) {
      const Key q{a, i >> (l - a), j >> (l - a), k >> (l - a)};
      if (s.count(q)) return q;
    }
    return {-1, 0, 0, 0};
  }
  bool wrap(int l, int (&p)[3]) const {  // periodic wrap; false outside a non-periodic domain
    for (int d = 0; d < 3; ++d) {
      const int N = m->bpd[d] << l;
      if (p[d] >= 0 && p[d] < N) continue;
      if (m->bc[d] != BC_PERIODIC) return false;
      p[d] = (p[d] % N + N) % N;
    }
    return true;
  }
  void split(const Key& k) {
    s.erase(k);
    for (int c = 0; c < 8; ++c) s.insert({k[0] + 1, 2 * k[1] + (c & 1), 2 * k[2] + ((c >> 1) & 1), 2 * k[3] + (c >> 2)});
  }
};
}  // namespace adapt_orc

// New leaf list (out: 4 ints per leaf, capacity 8*nb*4); returns the count.
extern "C" int orc_adapt_leaves(orc_mesh* m, const double* indicator, double rtol, double ctol, int32_t* out,
                                int cap) {
  using namespace adapt_orc;
  Leaves L{m, {}};
  for (int b = 0; b < m->nb; ++b) L.s.insert({m->level[b], m->idx[b][0], m->idx[b][1], m->idx[b][2]});
  for (int b = 0; b < m->nb; ++b)
    if (indicator[b] >= rtol && m->level[b] + 1 < m->level_max)
      L.split({m->level[b], m->idx[b][0], m->idx[b][1], m->idx[b][2]});
  // 2:1 balance: split any leaf more than one level coarser than a neighbour
  for (bool again = true; again;) {
    again = false;
    std::set<Key> todo;
    for (const Key& k : L.s)
      for (int e = 0; e < 27; ++e) {
        if (e == 13) continue;
        int p[3] = {k[1] + e % 3 - 1, k[2] + (e / 3) % 3 - 1, k[3] + e / 9 - 1};
        if (!L.wrap(k[0], p)) continue;
        const Key c = L.cover(k[0], p[0], p[1], p[2]);
        if (c[0] >= 0 && c[0] < k[0] - 1) todo.insert(c);
      }
    for (const Key& c : todo)
      if (L.s.count(c)) {
        L.split(c);
        again = true;
      }
  }
  // merging
  std::map<Key, int> votes;
  for (int b = 0; b < m->nb; ++b) {
    const Key k{m->level[b], m->idx[b][0], m->idx[b][1], m->idx[b][2]};
    if (k[0] == 0 || indicator[b] >= rtol || !(indicator[b] < ctol) || !L.s.count(k)) continue;
    ++votes[{k[0] - 1, k[1] >> 1, k[2] >> 1, k[3] >> 1}];
  }
  std::vector<Key> merge;
  for (const auto& kv : votes) {
    if (kv.second != 8) continue;
    const Key& P = kv.first;
    bool ok = true;
    for (int e = 0; e < 27 && ok; ++e) {
      if (e == 13) continue;
      int p[3] = {P[1] + e % 3 - 1, P[2] + (e / 3) % 3 - 1, P[3] + e / 9 - 1};
      if (!L.wrap(P[0], p)) continue;
      for (int c = 0; c < 8 && ok; ++c)
        ok = L.cover(P[0] + 1, 2 * p[0] + (c & 1), 2 * p[1] + ((c >> 1) & 1), 2 * p[2] + (c >> 2))[0] >= 0;
    }
    if (ok) merge.push_back(P);
  }
  for (const Key& P : merge) {
    for (int c = 0; c < 8; ++c) L.s.erase({P[0] + 1, 2 * P[1] + (c & 1), 2 * P[2] + ((c >> 1) & 1), 2 * P[3] + (c >> 2)});
    L.s.insert(P);
  }
  int n = 0;
  for (const Key& k : L.s) {
    if (n < cap)
      for (int q = 0; q < 4; ++q) out[4 * n + q] = k[q];
    ++n;
  }
  return n;
}

// Moves a field of m0 onto m1 (blocks in each mesh's own order).
extern "C" void orc_adapt_transfer(orc_mesh* m0, orc_mesh* m1, const double* f0, int ncomp, int vector_bc,
                                   double* f1) {
  const int64_t n0 = int64_t(m0->nb) * BN, n1 = int64_t(m1->nb) * BN;
#pragma omp parallel for schedule(dynamic, 4)
  for (int b = 0; b < m1->nb; ++b) {
    const int l = m1->level[b], i = m1->idx[b][0], j = m1->idx[b][1], k = m1->idx[b][2];
    const int same = m0->find(l, i, j, k);
    const int par = l > 0 ? m0->find(l - 1, i >> 1, j >> 1, k >> 1) : -1;
    if (same >= 0) {
      for (int c = 0; c < ncomp; ++c)
        for (int q = 0; q < BN; ++q) f1[c * n1 + int64_t(b) * BN + q] = f0[c * n0 + int64_t(same) * BN + q];
    } else if (par >= 0) {
      Lab lab(1, ncomp);
      fill_lab(*m0, f0, ncomp, 1, par, vector_bc != 0, lab);
      const int ox = i & 1, oy = j & 1, oz = k & 1;
      for (int z = 0; z < BS; ++z)
        for (int y = 0; y < BS; ++y)
          for (int x = 0; x < BS; ++x) {
            const int X = 4 * ox + x / 2, Y = 4 * oy + y / 2, Z = 4 * oz + z / 2;
            const double sx = (x % 2) ? 0.25 : -0.25, sy = (y % 2) ? 0.25 : -0.25, sz = (z % 2) ? 0.25 : -0.25;
            for (int c = 0; c < ncomp; ++c) {
              const double gx = 0.5 * (lab.at(c, X + 1, Y, Z) - lab.at(c, X - 1, Y, Z));
              const double gy = 0.5 * (lab.at(c, X, Y + 1, Z) - lab.at(c, X, Y - 1, Z));
              const double gz = 0.5 * (lab.at(c, X, Y, Z + 1) - lab.at(c, X, Y, Z - 1));
              f1[c * n1 + int64_t(b) * BN + cell(x, y, z)] = lab.at(c, X, Y, Z) + ((sx * gx + sy * gy) + sz * gz);
            }
          }
    } else {
      for (int Z = 0; Z < BS; ++Z)
        for (int Y = 0; Y < BS; ++Y)
          for (int X = 0; X < BS; ++X) {
            const int ch = m0->find(l + 1, 2 * i + X / 4, 2 * j + Y / 4, 2 * k + Z / 4);
            for (int c = 0; c < ncomp; ++c) {
              double s = 0.0;
              for (int e = 0; e < 8; ++e)
                s += f0[c * n0 + int64_t(ch) * BN + cell(2 * (X % 4) + (e & 1), 2 * (Y % 4) + ((e >> 1) & 1),
                                                      2 * (Z % 4) + (e >> 2))];
              f1[c * n1 + int64_t(b) * BN + cell(X, Y, Z)] = 0.125 * s;
            }
          }
    }
  }
}
