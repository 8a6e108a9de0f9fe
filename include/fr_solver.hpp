// fr_solver.hpp - C++ adapter with the reference `solver` method names over
// the C ABI of libfr_b200.so (include/fr_b200.h).
//
// A FlurryPP-style driver (reference: src/flurry.cpp:127-174) keeps its loop
//   Solver.setup(&params, params.order);  Solver.initializeSolution();
//   while (iter < iterMax) { iter++; Solver.update(); ... }
// and swaps `solver` for `fr::b200::Solver`, which reads the same deck.  The
// reference's fail-stop convention (FatalError = print + exit(1),
// include/error.hpp) becomes an exception carrying the library status.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "fr_b200.h"

namespace fr {
namespace b200 {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string &msg) : std::runtime_error(msg), code(code) {}
  int code;
};

class Solver {
 public:
  Solver() { fr_setup_opts_default(&opts_); }
  ~Solver() { fr_destroy(c_); }
  Solver(const Solver &) = delete;
  Solver &operator=(const Solver &) = delete;

  fr_setup_opts &options() { return opts_; }

  // solver::setup(input*, order, geo*) with input::readInputFile(deck)
  // (reference: src/solver.cpp:60-115, src/input.cpp:257-523)
  void setup(const std::string &deck) {
    fr_destroy(c_);
    c_ = nullptr;
    check(fr_create_from_deck(deck.c_str(), &opts_, &c_));
    check(fr_get_info(c_, &info_));
  }
  // solver::initializeSolution (src/solver.cpp:1892-1943): the deck's icType
  void initializeSolution() { check(fr_init_solution(c_, 0, nullptr, 0)); }
  // solver::update (src/solver.cpp:319-363)
  void update(bool pmgSource = false) { check(fr_update(c_, pmgSource ? 1 : 0)); }
  // solver::calcResidual (src/solver.cpp:366-445)
  void calcResidual(int step) { check(fr_calc_residual(c_, step)); }
  // solver::calcDt (src/solver.cpp:447-468)
  double calcDt() {
    double dt = 0.0;
    check(fr_calc_dt(c_, &dt));
    return dt;
  }
  // n steps with the steady-state step replayed as a CUDA graph
  void run(int n) { check(fr_run(c_, n)); }

  // U_spts / divF_spts[step] in the reference layout [spt][ele][field]
  std::vector<double> U_spts() {
    std::vector<double> u((size_t)info_.nSpts * info_.nEles * info_.nFields);
    check(fr_get_state(c_, u.data(), u.size()));
    return u;
  }
  void set_U_spts(const std::vector<double> &u) { check(fr_set_state(c_, u.data(), u.size())); }
  std::vector<double> divF_spts(int step) {
    std::vector<double> d((size_t)info_.nSpts * info_.nEles * info_.nFields);
    check(fr_get_residual(c_, step, d.data(), d.size()));
    return d;
  }
  // writeResidual's norm of divF_spts[0] (src/output.cpp:1011-1090)
  std::vector<double> residualNorm(int resType) {
    std::vector<double> r(info_.nFields);
    check(fr_residual_norm(c_, resType, r.data(), info_.nFields));
    return r;
  }

  // writeData (src/output.cpp:43-58): ParaView or CSV per the deck's
  // plotType; checkpoint() snapshots the state so the file can be written
  // later while stepping goes on; readRestartFile (src/solver.cpp:1789-1890)
  void checkpoint() { check(fr_checkpoint(c_)); }
  void writeData(const char *path = nullptr) { check(fr_write_data(c_, path)); }
  void readRestartFile(const char *path = nullptr) { check(fr_read_restart(c_, path)); }

  // integrateError (src/solver.cpp:1945-2028), writeResidual's force
  // coefficients, computeMassFlux (testCase 2)
  std::vector<double> integrateError(int errorNorm = -1) {
    std::vector<double> e(info_.nFields);
    check(fr_integrate_error(c_, errorNorm, e.data(), info_.nFields));
    return e;
  }
  std::vector<double> wallForce() {
    std::vector<double> f(6);
    check(fr_wall_force(c_, f.data()));
    return f;
  }
  std::vector<double> massFlux(int errorNorm = -1) {
    std::vector<double> m(info_.nFields);
    check(fr_mass_flux(c_, errorNorm, m.data(), info_.nFields));
    return m;
  }

  const fr_info &info() {
    check(fr_get_info(c_, &info_));
    return info_;
  }
  fr_case *handle() { return c_; }

 private:
  void check(int st) {
    if (st != FR_OK) throw Error(st, c_ ? fr_last_error(c_) : "fr_b200: setup failed");
  }
  fr_setup_opts opts_;
  fr_case *c_ = nullptr;
  fr_info info_{};
};

}  // namespace b200
}  // namespace fr
