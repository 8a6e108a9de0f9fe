// Element partition and halo plan for running one case on several GPUs.
//
// The reference partitions the mesh with METIS (geo::partitionMesh,
// src/geo.cpp:2380-2470) and, per stage, exchanges the left traces of every
// face cut by the partition with the rank across it (mpiFace::communicate,
// src/mpiFace.cpp:122-134); each side then forms the common flux of that face
// as its own left side, with the received trace as the right state
// (mpiFace::getRightState, src/mpiFace.cpp:158-175).  METIS is not
// available here: the partition is a recursive coordinate bisection of the
// element centroids (deterministic, balanced to one element per split).
//
// The halo plan lists, for one part, every face point of a cut face as
// (peer part, the point's slot in this part's local numbering), in one order
// both sides of a cut agree on: by face, then by point in the face's left
// order.  A part packs its traces at the listed slots, in list order, into
// the send buffer for each peer; the k-th value it receives from that peer
// is then the trace at the same face point seen from the other side.
#include <algorithm>
#include <numeric>

#include "fr_host.hpp"

namespace fr {

namespace {

void rcb(const std::vector<double> &cen, int nd, std::vector<int> &ids, int first, int nparts,
         std::vector<int> &part) {
  if (nparts == 1 || ids.size() <= 1) {
    for (int e : ids) part[e] = first;
    return;
  }
  int axis = 0;
  double best = -1.0;
  for (int d = 0; d < nd; d++) {
    double lo = 1e300, hi = -1e300;
    for (int e : ids) {
      lo = std::min(lo, cen[(size_t)e * nd + d]);
      hi = std::max(hi, cen[(size_t)e * nd + d]);
    }
    if (hi - lo > best) best = hi - lo, axis = d;
  }
  std::sort(ids.begin(), ids.end(), [&](int a, int b) {
    const double ca = cen[(size_t)a * nd + axis], cb = cen[(size_t)b * nd + axis];
    return ca < cb || (ca == cb && a < b);
  });
  const int p1 = nparts / 2;
  const size_t cut = ids.size() * (size_t)p1 / (size_t)nparts;
  std::vector<int> left(ids.begin(), ids.begin() + cut), right(ids.begin() + cut, ids.end());
  rcb(cen, nd, left, first, p1, part);
  rcb(cen, nd, right, first + p1, nparts - p1, part);
}

}  // namespace

bool partition_elements(const Mesh &m, int nparts, std::vector<int> &part, std::string &err) {
  if (nparts < 1 || nparts > m.nEles) {
    err = "partition: parts must be between 1 and the element count";
    return false;
  }
  const int nd = m.nDims, nCorner = nd == 2 ? 4 : 8;  // corner vertices lead every node list
  std::vector<double> cen((size_t)m.nEles * nd, 0.0);
  for (int e = 0; e < m.nEles; e++)
    for (int v = 0; v < nCorner; v++)
      for (int d = 0; d < nd; d++)
        cen[(size_t)e * nd + d] += m.xv[(size_t)m.c2v[(size_t)e * m.nNodes + v] * nd + d] / nCorner;
  std::vector<int> ids(m.nEles);
  std::iota(ids.begin(), ids.end(), 0);
  part.assign(m.nEles, 0);
  rcb(cen, nd, ids, 0, nparts, part);
  return true;
}

bool halo_plan(const Mesh &m, const std::vector<Face> &faces, int nPF, const std::vector<int> &part, int rank,
               std::vector<int> &owned, std::vector<int> &peer, std::vector<long long> &slot, std::string &err) {
  if ((int)part.size() != m.nEles) {
    err = "halo plan: partition size differs from the element count";
    return false;
  }
  owned.clear();
  std::vector<int> local(m.nEles, -1);
  for (int e = 0; e < m.nEles; e++)
    if (part[e] == rank) {
      local[e] = (int)owned.size();
      owned.push_back(e);
    }
  const long long nOwned = (long long)owned.size();
  peer.clear();
  slot.clear();
  for (const Face &f : faces) {
    if (f.eR < 0 || part[f.eL] == part[f.eR]) continue;
    const bool mineL = part[f.eL] == rank, mineR = part[f.eR] == rank;
    if (!mineL && !mineR) continue;
    for (int j = 0; j < nPF; j++) {
      if (mineL) {
        peer.push_back(part[f.eR]);
        slot.push_back((long long)(f.locL * nPF + j) * nOwned + local[f.eL]);
      } else {
        peer.push_back(part[f.eL]);
        slot.push_back((long long)f.fptR[j] * nOwned + local[f.eR]);
      }
    }
  }
  return true;
}

}  // namespace fr
