// Exercises the C++ mirror (include/topopt_b200.hpp) the way the
// reference's Main.cpp drives TopOpt: BCs, FEInitialize, MatIntFnc,
// FEAssemble, FESolve, Compliance and Volume.  Prints one line:
//   <status> <iterations> <compliance> <volume> <sum dC/dx> <sum dV/dx>
#include <cstdio>
#include <vector>

#include "topopt_b200.hpp"

int main() {
  tpo::TopOpt t({12, 6, 6}, {1.0, 1.0, 1.0}, 1.0, 0.3, 1.5, 2);
  if (!t.ok()) {
    std::printf("create failed: %s\n", t.last_error().c_str());
    return 2;
  }
  const double big = 1e10, tiny = 1e-10;
  const std::array<double, 6> open = {-1e30, 1e30, -1e30, 1e30, -1e30, 1e30};
  if (t.Set_BC({0, 0, 0}, {tiny, big, big}, open, {1, 1, 1}, tpo::SUPPORT) ||
      t.Set_BC({12, 0, 0}, {tiny, big, tiny}, open, {0, 0, -1.0 / 7}, tpo::LOAD))
    return 3;
  std::vector<double> x(t.nElem);
  for (int64_t e = 0; e < t.nElem; ++e) x[e] = 0.1 + 0.9 * ((e * 7919) % 101) / 100.0;
  if (t.FEInitialize() || t.MatIntFnc(x) || t.FEAssemble() || t.FESolve()) {
    std::printf("FE failed: %s\n", t.last_error().c_str());
    return 4;
  }
  tpo::Compliance c({1.0}, 0.0, 1.0, true);
  tpo::Volume v({0.3}, 0.0, 1.0, false);
  if (c.Compute(t) || v.Compute(t)) return 5;
  double sc = 0, sv = 0;
  for (double g : c.gradient) sc += g;
  for (double g : v.gradient) sv += g;
  // MMA::Update both ways: OCsub with the volume constraint alone, MMAsub
  // with it and mean(x) <= 0.35 over the first half of the elements
  const int64_t n = t.nElem, h = n / 2;
  tpo::MMA oc(t);
  oc.Set_Values(x);
  if (oc.Update(c.gradient, {v.value}, v.gradient)) return 6;
  double xh = 0, s_oc = 0, s_mma = 0;
  for (int64_t e = 0; e < h; ++e) xh += x[e] / h;
  std::vector<double> dg(2 * n, 0.0);
  for (int64_t e = 0; e < n; ++e) dg[e] = v.gradient[e];
  for (int64_t e = 0; e < h; ++e) dg[n + e] = 1.0 / h;
  tpo::MMA mma(t);
  mma.Set_Values(x);
  if (mma.Update(c.gradient, {v.value, xh - 0.35}, dg) || mma.Get_m() != 2) return 7;
  for (int64_t e = 0; e < n; ++e) {
    s_oc += oc.Get_x()[e];
    s_mma += mma.Get_x()[e];
  }
  std::printf("%d %d %.15g %.15g %.15g %.15g %.15g %.15g %.15g %.15g\n", t.KUF_reason,
              t.info.iterations, c.values0, v.values0, sc, sv, oc.Change, s_oc, mma.Change,
              s_mma);
  return t.KUF_reason == 0 ? 0 : 1;
}
