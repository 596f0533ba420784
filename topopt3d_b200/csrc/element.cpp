// Host-side element constants: the hex8 element stiffness K0 and its modal
// (Hadamard-basis) form used by the matrix-free kernels, and the density
// filter template.
#include <cmath>
#include <cstring>

#include "tpo_internal.h"

namespace tpo {

namespace {

// reference local node numbering of a hex8 (FEAnalysis.cpp:955-986):
// (---),(+--),(++-),(-+-),(--+),(+-+),(+++),(-++)
constexpr int kLocalSign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1},
                                  {-1, 1, -1},  {-1, -1, 1}, {1, -1, 1},
                                  {1, 1, 1},    {-1, 1, 1}};
// lexicographic corner l = bx + 2by + 4bz -> reference local node
constexpr int kLexToLocal[8] = {0, 1, 3, 2, 4, 5, 7, 6};

// (mode q, component c) pairs of the modal blocks, in packing order
struct BlockDef {
  int size;
  int q[3], c[3];
};
constexpr BlockDef kBlocks[] = {
    {3, {1, 2, 4}, {0, 1, 2}}, {2, {1, 2, 0}, {1, 0, 0}},
    {2, {1, 4, 0}, {2, 0, 0}}, {2, {2, 4, 0}, {2, 1, 0}},
    {2, {3, 6, 0}, {0, 2, 0}}, {2, {3, 5, 0}, {1, 2, 0}},
    {2, {6, 5, 0}, {1, 0, 0}}, {3, {3, 6, 5}, {2, 0, 1}},
    {1, {7, 0, 0}, {0, 0, 0}}, {1, {7, 0, 0}, {1, 0, 0}},
    {1, {7, 0, 0}, {2, 0, 0}},
};

double det3(const double a[9]) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) -
         a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// K0 = sum_q W_q B_q^T D B_q detJ over 2x2x2 Gauss points at +-1/sqrt(3),
// W = 1 (LocalK, FEAnalysis.cpp:869-892; B in Voigt order
// [xx,yy,zz,xy,yz,xz] with engineering shears, AssignB :1024-1046;
// D from RecMesh.cpp:453-462).
void element_stiffness(const double dx[3], double E0, double nu,
                       double K0[576]) {
  const double lam_c = E0 / ((1 + nu) * (1 - 2 * nu));
  const double G = E0 / (2 * (1 + nu));
  double D[6][6] = {};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[i][j] = (i == j) ? (1 - nu) * lam_c : nu * lam_c;
  D[3][3] = D[4][4] = D[5][5] = G;

  std::memset(K0, 0, 576 * sizeof(double));
  const double g = 1.0 / std::sqrt(3.0);
  for (int q = 0; q < 8; ++q) {
    const double xi[3] = {kLocalSign[q][0] * g, kLocalSign[q][1] * g,
                          kLocalSign[q][2] * g};
    double dN[3][8];
    for (int n = 0; n < 8; ++n) {
      const double a = kLocalSign[n][0], b = kLocalSign[n][1],
                   c = kLocalSign[n][2];
      dN[0][n] = a * (1 + b * xi[1]) * (1 + c * xi[2]) / 8.0;
      dN[1][n] = b * (1 + a * xi[0]) * (1 + c * xi[2]) / 8.0;
      dN[2][n] = c * (1 + a * xi[0]) * (1 + b * xi[1]) / 8.0;
    }
    // J = dN * coords; for a box element J is diagonal dx/2
    double J[9] = {};
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc)
        for (int n = 0; n < 8; ++n)
          J[3 * r + cc] += dN[r][n] * (kLocalSign[n][cc] > 0 ? dx[cc] : 0.0);
    const double detJ = det3(J);
    double Ji[9];
    Ji[0] = (J[4] * J[8] - J[5] * J[7]) / detJ;
    Ji[1] = (J[2] * J[7] - J[1] * J[8]) / detJ;
    Ji[2] = (J[1] * J[5] - J[2] * J[4]) / detJ;
    Ji[3] = (J[5] * J[6] - J[3] * J[8]) / detJ;
    Ji[4] = (J[0] * J[8] - J[2] * J[6]) / detJ;
    Ji[5] = (J[2] * J[3] - J[0] * J[5]) / detJ;
    Ji[6] = (J[3] * J[7] - J[4] * J[6]) / detJ;
    Ji[7] = (J[1] * J[6] - J[0] * J[7]) / detJ;
    Ji[8] = (J[0] * J[4] - J[1] * J[3]) / detJ;
    double dX[3][8];
    for (int r = 0; r < 3; ++r)
      for (int n = 0; n < 8; ++n)
        dX[r][n] = Ji[3 * r] * dN[0][n] + Ji[3 * r + 1] * dN[1][n] +
                   Ji[3 * r + 2] * dN[2][n];
    double B[6][24] = {};
    for (int n = 0; n < 8; ++n) {
      B[0][3 * n] = dX[0][n];
      B[1][3 * n + 1] = dX[1][n];
      B[2][3 * n + 2] = dX[2][n];
      B[3][3 * n] = dX[1][n];
      B[3][3 * n + 1] = dX[0][n];
      B[4][3 * n + 1] = dX[2][n];
      B[4][3 * n + 2] = dX[1][n];
      B[5][3 * n] = dX[2][n];
      B[5][3 * n + 2] = dX[0][n];
    }
    for (int r = 0; r < 24; ++r)
      for (int cc = 0; cc < 24; ++cc) {
        double s = 0;
        for (int a = 0; a < 6; ++a)
          for (int b = 0; b < 6; ++b) s += B[a][r] * D[a][b] * B[b][cc];
        K0[24 * r + cc] += s * detJ;
      }
  }
}

}  // namespace

// Gauss-point gradients of the trilinear shape functions of a box element
// for the stress stiffness: corner l (lexicographic, sign s_d = +1 when bit
// d of l is set), Gauss point q at xi_d = s_d(q) / sqrt(3);
// dN_l/dx_a = s_a(l)/8 prod_{d != a} (1 + s_d(l) xi_d) * 2/dx_a and
// detJ = dx dy dz / 8 (the box-element case of FEAnalysis.cpp:869-990)
static void build_ks_constants(Ctx &c) {
  const double g = 1.0 / std::sqrt(3.0);
  auto sg = [](int l, int d) { return ((l >> d) & 1) ? 1.0 : -1.0; };
  for (int q = 0; q < 8; ++q)
    for (int a = 0; a < 3; ++a)
      for (int l = 0; l < 8; ++l) {
        double v = sg(l, a) / 8.0 * 2.0 / c.prm.dx[a];
        for (int d = 0; d < 3; ++d)
          if (d != a) v *= 1.0 + sg(l, d) * sg(q, d) * g;
        c.ksc.g[q][a][l] = v;
      }
  const double E0 = c.prm.E0, nu = c.prm.nu;
  const double cc = E0 / ((1 + nu) * (1 - 2 * nu));
  c.ksc.t1 = (1 - nu) * cc;
  c.ksc.t3 = nu * cc;
  c.ksc.t2 = E0 / (2 * (1 + nu));
  c.ksc.detJ = c.prm.dx[0] * c.prm.dx[1] * c.prm.dx[2] / 8.0;
}

// Level-1 Galerkin blocks of an interior fine element: the fine element at
// offset i = (ax, ay, az) inside its coarse element has corner p at fine
// coordinate t_d = a_d + bit_d(p) in {0, 1, 2} from the coarse element's
// origin; the trilinear weight of coarse corner k is W[t][bit_d(k)] with
// W = {{1, 0}, {1/2, 1/2}, {0, 1}} per dimension (Interpolation.cpp:135,
// 157; interior rows need no normalisation).  GMi[i][ln][lm] =
// sum_{p,q} w(p->ln) w(q->lm) K0[p][q] (3x3 blocks, lexicographic corners).
static void build_galerkin_blocks(Ctx &c, const double Kl[24][24]) {
  static const double W[3][2] = {{1.0, 0.0}, {0.5, 0.5}, {0.0, 1.0}};
  for (int i = 0; i < 8; ++i) {
    double w[8][8];   // w[p][k]
    for (int p = 0; p < 8; ++p)
      for (int k = 0; k < 8; ++k) {
        double v = 1.0;
        for (int d = 0; d < 3; ++d)
          v *= W[((i >> d) & 1) + ((p >> d) & 1)][(k >> d) & 1];
        w[p][k] = v;
      }
    for (int ln = 0; ln < 8; ++ln)
      for (int lm = 0; lm < 8; ++lm)
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) {
            double v = 0.0;
            for (int p = 0; p < 8; ++p)
              for (int q = 0; q < 8; ++q)
                v += w[p][ln] * w[q][lm] * Kl[3 * p + r][3 * q + s];
            c.GMi_h[((i * 8 + ln) * 8 + lm) * 9 + 3 * r + s] = v;
          }
  }
}

int build_element_constants(Ctx &c) {
  element_stiffness(c.prm.dx, c.prm.E0, c.prm.nu, c.K0);
  build_ks_constants(c);
  // K0 in lexicographic corner order
  double Kl[24][24];
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b)
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s)
          Kl[3 * a + r][3 * b + s] =
              c.K0[24 * (3 * kLexToLocal[a] + r) + 3 * kLexToLocal[b] + s];
  for (int i = 0; i < 24; ++i) c.kd64.v[i] = Kl[i][i];
  build_galerkin_blocks(c, Kl);
  // Kh = T K T^T / 64 indexed (3q + c)
  auto sgn = [](int l, int q) {
    int s = 1;
    for (int d = 0; d < 3; ++d)
      if ((q >> d) & 1) s *= ((l >> d) & 1) ? 1 : -1;
    return s;
  };
  double Kh[24][24];
  double kmax = 0;
  for (int qa = 0; qa < 8; ++qa)
    for (int ca = 0; ca < 3; ++ca)
      for (int qb = 0; qb < 8; ++qb)
        for (int cb = 0; cb < 3; ++cb) {
          double s = 0;
          for (int la = 0; la < 8; ++la)
            for (int lb = 0; lb < 8; ++lb)
              s += sgn(la, qa) * sgn(lb, qb) * Kl[3 * la + ca][3 * lb + cb];
          Kh[3 * qa + ca][3 * qb + cb] = s / 64.0;
          kmax = std::fmax(kmax, std::fabs(s / 64.0));
        }
  bool covered[24][24] = {};
  int k = 0;
  for (const BlockDef &bd : kBlocks)
    for (int i = 0; i < bd.size; ++i)
      for (int j = 0; j < bd.size; ++j) {
        const int ri = 3 * bd.q[i] + bd.c[i], cj = 3 * bd.q[j] + bd.c[j];
        c.kh64.v[k] = Kh[ri][cj];
        c.kh32.v[k] = static_cast<float>(Kh[ri][cj]);
        covered[ri][cj] = true;
        ++k;
      }
  if (k != kNumKh) {
    c.err = "internal: modal block table has the wrong size";
    return TPO_E_UNSUPPORTED;
  }
  for (int i = 0; i < 24; ++i)
    for (int j = 0; j < 24; ++j)
      if (!covered[i][j] && std::fabs(Kh[i][j]) > 1e-12 * kmax) {
        c.err = "element stiffness does not decouple in the modal basis";
        return TPO_E_UNSUPPORTED;
      }
  return TPO_OK;
}

bool build_filter_taps(const int nel[3], const double dx[3], double R,
                       FilterTaps &taps) {
  // RecFilter (Filter.cpp:28-52): N = floor(R/dx) neighbours per side,
  // weight 1 - d/R for d < R (strict), template in (k, j, i) order which is
  // increasing column order of the assembled filter matrix.
  // offsets are stored as int8: refuse radii that do not fit (and
  // non-finite or non-positive input) before the conversion
  if (!std::isfinite(R) || !(R > 0)) return false;
  int N[3];
  for (int d = 0; d < 3; ++d) {
    if (!std::isfinite(dx[d]) || !(dx[d] > 0) || !(R / dx[d] <= 127.0)) return false;
    N[d] = static_cast<int>(R / dx[d]);
  }
  taps.n = 0;
  for (int k = -N[2]; k <= N[2]; ++k)
    for (int j = -N[1]; j <= N[1]; ++j)
      for (int i = -N[0]; i <= N[0]; ++i) {
        const double dist = std::sqrt(std::pow(i * dx[0], 2) +
                                      std::pow(j * dx[1], 2) +
                                      std::pow(k * dx[2], 2));
        if (!(dist < R)) continue;
        if (taps.n >= kMaxFilterTaps) return false;
        taps.off[taps.n][0] = static_cast<int8_t>(i);
        taps.off[taps.n][1] = static_cast<int8_t>(j);
        taps.off[taps.n][2] = static_cast<int8_t>(k);
        taps.w[taps.n] = 1 - dist / R;
        ++taps.n;
      }
  (void)nel;
  return taps.n > 0;
}

}  // namespace tpo
