/*
 * Row de-duplication for the timing build of the reference (oracle/_ref/
 * fr_ref_harness_omp), so that its mesh setup at 32^3 hexes takes about two
 * minutes instead of about twenty.
 *
 * The reference's matrix<int>::unique (src/matrix.cpp:668-695) compares each
 * row with every earlier row: O(n^2) in the rows.  geo::processConn3D calls it
 * on the 6*nEles element faces and 12*nEles element edges (src/geo.cpp:429-430),
 * which at 32^3 hexes is 393,216 edge rows.  This definition returns the same
 * result, by a hash of the rows instead of the pairwise search:
 *   - out holds the distinct rows in order of first occurrence;
 *   - iRow[i] is the row of out equal to row i.
 * As an explicit specialisation it takes the place, at link time, of the
 * member the reference's explicit instantiation of matrix<int> provides.
 *
 * It is used only by mesh setup, before and outside the timed solver::update
 * loop; the parity oracle (fr_ref_harness, -O2) keeps the reference's own
 * function.  tests/test_oracle.py checks that both builds produce the same
 * face connectivity.
 *
 * Test infrastructure: never linked into the product library.
 */
#include <string>
#include <unordered_map>
#include <vector>

#include "matrix.hpp"

template <>
void matrix<int>::unique(matrix<int> &out, std::vector<int> &iRow) {
  const size_t n = this->dims[0], w = this->dims[1];
  iRow.assign(n, -1);
  std::unordered_map<std::string, int> first;
  first.reserve(2 * n + 1);
  std::vector<int> rows;
  int nOut = 0;
  for (size_t i = 0; i < n; i++) {
    const int *row = this->data.data() + i * w;
    std::string key(reinterpret_cast<const char *>(row), w * sizeof(int));
    auto it = first.find(key);
    if (it != first.end()) {
      iRow[i] = it->second;
      continue;
    }
    first.emplace(std::move(key), nOut);
    rows.insert(rows.end(), row, row + w);
    iRow[i] = nOut++;
  }
  out.setup(nOut, w);
  for (size_t k = 0; k < rows.size(); k++) out.data[k] = rows[k];
}
