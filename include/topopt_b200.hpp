// topopt_b200.hpp -- header-only C++ mirror of the darinpeetz/TopOpt3D
// finite-element call surface over the C ABI in topopt_b200.h.
//
// A reference caller keeps its call sequence (Main.cpp:138-169):
//
//   tpo::TopOpt t({nx, ny, nz}, {dx, dy, dz}, E0, Nu0, rmin, levels);
//   t.Set_BC(center, radius, limits, values, tpo::SUPPORT);   // Inputs.cpp:105
//   t.FEInitialize();                                          // FEAnalysis.cpp:215
//   t.MatIntFnc(x);                     // Material_Interpolation.cpp:20
//   t.FEAssemble();                     // FEAnalysis.cpp:432
//   t.FESolve();                        // FEAnalysis.cpp:507
//   tpo::Compliance c({1.0}, 0, 1, true);
//   c.Compute(t);                       // Functions.cpp:39
//
// Methods return the library status as the reference returns a
// PetscErrorCode: 0 on success, negative on error (message in
// last_error()), positive when the solver stopped without converging
// (KUF_reason, FEAnalysis.cpp:677).  Vectors are std::vector<double> on the
// host in the reference numbering.
#ifndef TOPOPT_B200_HPP
#define TOPOPT_B200_HPP

#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "topopt_b200.h"

namespace tpo {

enum BCTYPE { SUPPORT = TPO_BC_SUPPORT, LOAD = TPO_BC_LOAD };

class TopOpt {
 public:
  TopOpt(std::array<int, 3> nel, std::array<double, 3> dx, double E0,
         double Nu0, double rmin, int mg_levels = 0) {
    tpo_mesh_params p{};
    for (int d = 0; d < 3; ++d) {
      p.nel[d] = nel[d];
      p.dx[d] = dx[d];
    }
    p.E0 = E0;
    p.nu = Nu0;
    p.rmin = rmin;
    p.mg_levels = mg_levels;
    status_ = tpo_create(&p, &ctx_);
    if (ctx_) tpo_sizes(ctx_, &nElem, &nNode, &levels);
    tpo_default_solve_opts(&opts);
    tpo_default_eig_opts(&eig);
  }
  ~TopOpt() { tpo_destroy(ctx_); }
  // TopOpt::LoadMesh (RecMesh.cpp:34-412): a problem from a MeshOut folder
  // of a structured box (null on failure; tpo_last_error(NULL) says why)
  static std::unique_ptr<TopOpt> LoadMesh(const std::string &folder, double E0, double Nu0,
                                          double rmin, int mg_levels = 0,
                                          int index_bytes = 4) {
    tpo_mesh_params p{};
    p.E0 = E0;
    p.nu = Nu0;
    p.rmin = rmin;
    p.mg_levels = mg_levels;
    tpo_ctx *h = nullptr;
    if (tpo_load_mesh(folder.c_str(), &p, index_bytes, &h) != 0) return nullptr;
    return std::unique_ptr<TopOpt>(new TopOpt(h));
  }
  TopOpt(const TopOpt &) = delete;
  TopOpt &operator=(const TopOpt &) = delete;

  bool ok() const { return ctx_ != nullptr && status_ >= 0; }
  std::string last_error() const {
    return ctx_ ? tpo_last_error(ctx_) : "context creation failed";
  }
  tpo_ctx *handle() { return ctx_; }

  int Set_BC(std::array<double, 3> center, std::array<double, 3> radius,
             std::array<double, 6> limits, std::array<double, 3> values,
             BCTYPE type) {
    int64_t n = 0;
    return tpo_add_bc(ctx_, type, center.data(), radius.data(), limits.data(),
                      values.data(), &n);
  }
  int FEInitialize() { return tpo_fe_initialize(ctx_); }
  int MatIntFnc(const std::vector<double> &design) {
    return tpo_mat_int_fnc(ctx_, design.data(), penal, eps, TPO_MEM_HOST);
  }
  int FEAssemble() { return tpo_fe_assemble(ctx_, &opts); }
  int FESolve() {
    KUF_reason = tpo_fe_solve(ctx_, &opts, &info);
    return KUF_reason < 0 ? KUF_reason : 0;
  }
  // Chain_Filter (Material_Interpolation.cpp:150-187) with vdMin <= 0:
  // dfdV <- P^T dfdV and dfdE <- P^T dfdE, in place; either may be null
  int Chain_Filter(std::vector<double> *dfdV, std::vector<double> *dfdE) {
    for (std::vector<double> *v : {dfdV, dfdE}) {
      if (!v) continue;
      std::vector<double> out(v->size());
      int rc = tpo_filter(ctx_, v->data(), out.data(), 1, TPO_MEM_HOST);
      if (rc) return rc;
      v->swap(out);
    }
    return 0;
  }
  // Stability (Buckling.cpp:15-361): Ks from the current U, then the
  // eig.nev largest eigenvalues of Ks phi = lambda K phi (descending)
  int StressFnc() { return tpo_ks_assemble(ctx_); }
  int Buckling(std::vector<double> &lambda) {
    lambda.assign(eig.nev, 0.0);
    const int rc = tpo_buckling(ctx_, &eig, lambda.data(), nullptr, TPO_MEM_HOST,
                                &eig_info);
    return rc < 0 ? rc : 0;
  }
  // Stability::Function with its gradient (Buckling.cpp:15-272): the
  // eigenpairs, value = (sum lambda^p)^(1/p) and dvalue/dx through one
  // adjoint solve per eigenpair (solved with `opts`)
  int BucklingGradient(std::vector<double> &lambda, double p, double *value,
                       std::vector<double> &dvdx) {
    lambda.assign(eig.nev, 0.0);
    std::vector<double> phi((size_t)eig.nev * 3 * nNode);
    int rc = tpo_buckling(ctx_, &eig, lambda.data(), phi.data(), TPO_MEM_HOST, &eig_info);
    if (rc < 0) return rc;
    dvdx.assign(nElem, 0.0);
    rc = tpo_buckling_sensitivity(ctx_, eig.nev, lambda.data(), phi.data(), p, &opts, value,
                                  dvdx.data(), nullptr, TPO_MEM_HOST, nullptr);
    return rc < 0 ? rc : 0;
  }
  // TopOpt::MeshOut (TopOpt.cpp:97-359) and PrintVals (:445-508); modes
  // are 3*nNode x n column-major
  int MeshOut(const std::string &folder = ".", double rmax = 3.0, int index_bytes = 4) {
    return tpo_mesh_out(ctx_, folder.c_str(), rmax, index_bytes);
  }
  int PrintVals(const std::string &name_suffix, const std::string &folder = ".",
                const std::vector<double> &phiB = {}, const std::vector<double> &phiD = {},
                int index_bytes = 4) {
    const int64_t nd = 3 * nNode;
    return tpo_print_vals(ctx_, folder.c_str(), name_suffix.c_str(),
                          phiB.empty() ? nullptr : phiB.data(), (int32_t)(phiB.size() / nd),
                          phiD.empty() ? nullptr : phiD.data(), (int32_t)(phiD.size() / nd),
                          index_bytes);
  }
  std::vector<double> get(const char *which) const {
    const bool nodal = which[0] == 'U' || which[0] == 'F';
    std::vector<double> out(nodal ? 3 * nNode : nElem);
    tpo_get_vector(ctx_, which, out.data(), TPO_MEM_HOST);
    return out;
  }

  int64_t nElem = 0, nNode = 0;
  int32_t levels = 0;
  double penal = 3.0;
  double eps = 1e-10;            // Material_Interpolation.cpp:28
  tpo_solve_opts opts{};
  tpo_solve_info info{};
  tpo_eig_opts eig{};
  tpo_eig_info eig_info{};
  int KUF_reason = 0;

 private:
  explicit TopOpt(tpo_ctx *h) : ctx_(h) {
    tpo_sizes(ctx_, &nElem, &nNode, &levels);
    tpo_default_solve_opts(&opts);
    tpo_default_eig_opts(&eig);
  }
  tpo_ctx *ctx_ = nullptr;
  int status_ = 0;
};

// Function_Base (Functions.h:16-63, Functions.cpp:39-62)
class Function_Base {
 public:
  Function_Base(std::vector<double> values, double min_val, double max_val,
                bool objective, bool calc_gradient = true)
      : weights(std::move(values)), min_val(min_val), max_val(max_val),
        objective(objective), calc_gradient(calc_gradient) {}
  virtual ~Function_Base() = default;
  // Function_Base::name[func_type] (Functions.cpp:5)
  virtual const char *name() const { return "Function"; }

  int Compute(TopOpt &t) {
    int rc = Function(t);
    if (rc) return rc;
    const double w = weights.empty() ? 1.0 : weights[0];
    const double range = max_val - min_val;
    value = (objective ? w : 1.0) * (values0 - min_val) - (objective ? 0.0 : w);
    value /= range;
    gradient.resize(gradients.size());
    for (size_t i = 0; i < gradients.size(); ++i)
      gradient[i] = (objective ? w : 1.0) * gradients[i] / range;
    return 0;
  }

  std::vector<double> weights;
  double min_val, max_val;
  bool objective, calc_gradient;
  double values0 = 0.0, value = 0.0;
  std::vector<double> gradients, gradient;

 protected:
  virtual int Function(TopOpt &t) = 0;
};

// Compliance::Function (Compliance.cpp:15-57)
class Compliance : public Function_Base {
 public:
  using Function_Base::Function_Base;
  const char *name() const override { return "Compliance"; }

 protected:
  int Function(TopOpt &t) override {
    gradients.assign(calc_gradient ? t.nElem : 0, 0.0);
    return tpo_compliance(t.handle(), &values0,
                          calc_gradient ? gradients.data() : nullptr, nullptr,
                          TPO_MEM_HOST);
  }
};

// Volume::Function (Volume.cpp:15-41); constraint values are pre-scaled by
// the range as the input parser does (Inputs.cpp:554-557)
class Volume : public Function_Base {
 public:
  Volume(std::vector<double> values, double min_val, double max_val,
         bool objective, bool calc_gradient = true)
      : Function_Base(scale(values, min_val, max_val, objective), min_val,
                      max_val, objective, calc_gradient) {}
  const char *name() const override { return "Volume"; }

 protected:
  static std::vector<double> scale(std::vector<double> v, double lo, double hi,
                                   bool objective) {
    if (!objective)
      for (double &x : v) x *= hi - lo;
    return v;
  }
  int Function(TopOpt &t) override {
    gradients.assign(calc_gradient ? t.nElem : 0, 0.0);
    return tpo_volume(t.handle(), &values0,
                      calc_gradient ? gradients.data() : nullptr, TPO_MEM_HOST);
  }
};

// Stability::Function (Buckling.cpp:15-272): the buckling eigenvalues of
// Ks phi = lambda K phi aggregated as (sum lambda^p)^(1/p), p = 8, and with
// calc_gradient its design gradient
class Stability : public Function_Base {
 public:
  using Function_Base::Function_Base;
  const char *name() const override { return "Stability"; }

 protected:
  int Function(TopOpt &t) override {
    const double p = 8.0;
    if (int rc = t.StressFnc()) return rc;
    std::vector<double> lambda;
    if (calc_gradient) return t.BucklingGradient(lambda, p, &values0, gradients);
    gradients.clear();
    if (int rc = t.Buckling(lambda)) return rc;
    double s = 0.0;
    for (double l : lambda) s += std::pow(l, p);
    values0 = std::pow(s, 1.0 / p);
    return 0;
  }
};

// Frequency::Function (Dynamic.cpp:18-171): the largest eigenvalues of
// M phi = lambda K phi (the lowest natural frequencies) with the lumped
// mass of DiagMassFnc, aggregated as (sum lambda^p)^(1/p), p = 8, and with
// calc_gradient its design gradient
class Frequency : public Function_Base {
 public:
  Frequency(std::vector<double> values, double min_val, double max_val, bool objective,
            bool calc_gradient, int nvals, double density)
      : Function_Base(std::move(values), min_val, max_val, objective, calc_gradient),
        nvals(nvals), density(density) {}
  const char *name() const override { return "Frequency"; }
  int nvals;
  double density;
  std::vector<double> lambda;

 protected:
  int Function(TopOpt &t) override {
    lambda.assign(32, 0.0);
    int32_t nconv = 0;
    gradients.assign(calc_gradient ? t.nElem : 0, 0.0);
    const int rc = tpo_frequency(t.handle(), nvals, density, nullptr, &t.eig, 8.0,
                                 lambda.data(), &nconv, &values0,
                                 calc_gradient ? gradients.data() : nullptr, TPO_MEM_HOST,
                                 &t.eig_info);
    lambda.resize(nconv);
    return rc < 0 ? rc : 0;
  }
};

// MMA (MMA.h:14-100): the optimiser object of the reference, on the GPU of
// `t`.  Update (MMA.cpp:62-100) takes OCsub (OCeta = 0.5) for fewer than
// two constraints and MMAsub with DualSolve otherwise, with Set_m's
// constants a0 = b0 = 1, a = 0, c = 1000, d = 1.  dgdx is n x m
// column-major, as an Eigen::MatrixXd stores it.
class MMA {
 private:
  TopOpt &t_;
  int m_ = 0;

 public:
  explicit MMA(TopOpt &t)
      : t_(t), xval(t.nElem, 0.0), xold1(t.nElem, 0.0), xold2(t.nElem, 0.0),
        low(t.nElem, 0.0), upp(t.nElem, 1.0), xmin(t.nElem, 0.0), xmax(t.nElem, 1.0) {
    tpo_default_mma_opts(&opts);   // Set_Defaults (MMA.h:21-23)
  }
  void Set_Lower_Bound(std::vector<double> v) { xmin = std::move(v); }
  void Set_Upper_Bound(std::vector<double> v) { xmax = std::move(v); }
  void Set_Iter_Limit_Min(unsigned v) { miniter = v; }
  void Set_Iter_Limit_Max(unsigned v) { maxiter = v; }
  void Set_Change_Limit(double v) { minchange = v; }
  void Set_Step_Limit(double v) { opts.move = v; }
  void Set_Values(const std::vector<double> &x) { xval = xold1 = xold2 = x; }
  void Set_It(unsigned it) { iter = it; }
  void Restart() { fresh_start = true; }
  std::vector<double> &Get_x() { return xval; }
  unsigned &Get_It() { return iter; }
  int64_t Get_n() const { return t_.nElem; }
  int Get_m() const { return m_; }
  bool Check() { return Check_Conv() || Check_It(); }
  bool Check_Conv() const { return iter > miniter && Change < minchange; }
  bool Check_It() { return ++iter >= maxiter; }

  int Update(std::vector<double> dfdx, const std::vector<double> &g,
             const std::vector<double> &dgdx) {
    m_ = (int)g.size();
    const int64_t n = t_.nElem;
    if (m_ < 1 || (int64_t)dfdx.size() != n || (int64_t)dgdx.size() != n * m_ ||
        (int64_t)xval.size() != n)
      return TPO_E_ARG;
    if (m_ < 2)
      return tpo_oc_update(t_.handle(), xval.data(), xmin.data(), xmax.data(), dfdx.data(),
                           g[0], dgdx.data(), opts.move, &Change, TPO_MEM_HOST);
    int32_t fresh = fresh_start ? 1 : 0;
    const int rc = tpo_mma_update(t_.handle(), &opts, (int32_t)iter, &fresh, m_, xval.data(),
                                  xold1.data(), xold2.data(), low.data(), upp.data(),
                                  xmin.data(), xmax.data(), dfdx.data(), g.data(),
                                  dgdx.data(), &Change, TPO_MEM_HOST);
    fresh_start = fresh != 0;
    return rc;
  }

  tpo_mma_opts opts{};
  std::vector<double> xval, xold1, xold2, low, upp, xmin, xmax;
  double Change = 1.0;
  unsigned iter = 0, miniter = 0, maxiter = 50;
  double minchange = 0.0;
  bool fresh_start = true;
};

// TopOpt::StepOut's Output.txt entry (TopOpt.cpp:386-401)
inline void StepOut(std::FILE *out, double f, const std::vector<double> &cons, int it,
                    const std::vector<Function_Base *> &functions) {
  std::fprintf(out, "Iteration number: %u\n", (unsigned)it);
  std::fprintf(out, "Objective: %1.6g\n", f);
  std::fprintf(out, "Constraints:\n");
  for (double c : cons) std::fprintf(out, "\t%1.12g\t", c);
  std::fprintf(out, "\nAll function values:\n");
  for (const Function_Base *fn : functions)
    std::fprintf(out, "\t%12s: %1.8g\n", fn->name(), fn->value);
  std::fprintf(out, "\n");
}

// TopOpt::ResultOut (TopOpt.cpp:415-435): the stiffness-to-volume line,
// then PrintVals with the suffix _pen<penal> into `folder`
inline int ResultOut(std::FILE *out, TopOpt &t, int it, const std::string &folder = ".") {
  double Esum = 0, Vsum = 0;
  for (double v : t.get("E")) Esum += v;
  for (double v : t.get("rho")) Vsum += v;
  std::fprintf(out,
               "************************************************\nAfter %4i iterations "
               "with a penalty of %1.4g the\nratio of stiffness sum to volume sum is "
               "%1.4g\n************************************************\n\n",
               it, t.penal, Esum / Vsum);
  char sfx[30];
  std::snprintf(sfx, sizeof sfx, "_pen%1.4g", t.penal);
  return t.PrintVals(sfx, folder);
}

}  // namespace tpo

#endif  // TOPOPT_B200_HPP
