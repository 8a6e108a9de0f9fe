// Minimal FlurryPP-style driver on the B200 path (reference: src/flurry.cpp:71-188):
// read a deck, set up, apply the deck's initial condition (or its restart
// file), take N steps of update(), printing the residual norm every `freq`
// steps and at the end.  With WRITE = 1 it also writes the deck's solution
// files like the reference's loop: at the start, every plotFreq iterations
// (taken as checkpoints, written while the next steps run) and at the end.
//
// With ERR = 1 it ends with the error integrals of a testCase 1 deck.
//
//   flurry_b200 DECK NSTEPS [FREQ [WRITE [PLOTFREQ [ERR]]]]
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "../../include/fr_solver.hpp"

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s DECK NSTEPS [FREQ]\n", argv[0]);
    return 2;
  }
  const int nsteps = std::atoi(argv[2]);
  const int freq = argc > 3 ? std::atoi(argv[3]) : 10;
  const bool write = argc > 4 && std::atoi(argv[4]) != 0;
  const int plotFreq = argc > 5 ? std::atoi(argv[5]) : 100;
  const bool err = argc > 6 && std::atoi(argv[6]) != 0;
  try {
    fr::b200::Solver S;
    S.setup(argv[1]);
    S.initializeSolution();
    const fr_info &inf = S.info();
    std::printf("case: nDims %d order %d nEles %d nSpts %d nFields %d\n", inf.nDims, inf.order, inf.nEles,
                inf.nSpts, inf.nFields);
    if (write) S.writeData();
    const long long iter0 = S.info().iter;
    bool pending = false;
    for (int iter = 1; iter <= nsteps; iter++) {
      S.update();
      if (write && pending) {  // the previous checkpoint's copy overlapped this step
        S.writeData();
        pending = false;
      }
      if (write && ((iter0 + iter) % plotFreq == 0 || iter == nsteps)) {
        S.checkpoint();
        pending = true;
      }
      if (iter % freq == 0 || iter == nsteps) {
        auto r = S.residualNorm(2);
        std::printf("iter %6d  time %.10e  res", iter, S.info().time);
        for (double v : r) std::printf(" %.10e", v);
        std::printf("\n");
      }
    }
    if (pending) S.writeData();
    if (err) {  // writeAllError for testCase 1 (src/output.cpp:1212-1227)
      const char *what[3] = {"Integrated conservation error", "Integral L1 error", "Integral L2 error"};
      for (int n = 0; n < 3; n++) {
        auto e = S.integrateError(n);
        std::printf("%s:\n%-8lld Err ", what[n], S.info().iter);
        for (double v : e) std::printf(" %.6e", std::fabs(v));
        std::printf("\n");
      }
    }
  } catch (const fr::b200::Error &e) {
    std::fprintf(stderr, "fr_b200 error %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}
