// Domain decomposition of the element set and the per-rank halo plan for the
// face-trace exchange of a multi-rank run.
//
// The reference splits the elements into contiguous ranges (DomainDecomp,
// src/SELF_Mesh.f90:2159-2177) and exchanges each side shared with another
// rank with one MPI_IRECV / MPI_ISEND pair tagged by the global side id,
// followed by ApplyFlip (src/SELF_MappedData.f90:3323-3443).  Here a rank's
// off-rank neighbours become halo elements appended after its own in the
// engine's trace cache: the rank's sideInfo points those sides at the halo
// element and the neighbour's side, so the fused stage kernel applies the flip
// itself and needs no change.  The exchange moves, per peer, one packed buffer
// of trace blocks in an order both ranks derive independently (the shared
// faces sorted by their lower global (element, side) endpoint).
#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "selfgpu_internal.h"

using namespace selfgpu;

extern "C" {

// HOPR Meshformat Algorithm 4 as in DomainDecomp: the first nElems mod
// nDomains ranks take one extra element.  offsetElem has nDomains + 1 entries.
int selfgpu_domain_decomp(int nElems, int nDomains, int* offsetElem) {
  if (nElems < 1 || nDomains < 1 || nDomains > nElems || !offsetElem)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_domain_decomp: bad arguments");
  const int nLocal = nElems / nDomains;
  const int remain = nElems - nLocal * nDomains;
  for (int d = 0; d < nDomains; ++d) offsetElem[d] = d * nLocal + std::min(d, remain);
  offsetElem[nDomains] = nElems;
  return SELFGPU_OK;
}

// ElemToRank (src/SELF_Mesh.f90:2179-2215, HOPR Algorithm 7): the rank whose
// range (offsetElem(d), offsetElem(d+1)] holds the 1-based elemID, by the
// reference's bisection (checks the two end ranks, then at most
// floor(log2(nDomains)) + 1 halvings).
int selfgpu_elem_to_rank(int nDomains, const int* offsetElem, int elemID, int* domain) {
  if (nDomains < 1 || !offsetElem || !domain) return set_error(SELFGPU_ERR_ARG, "selfgpu_elem_to_rank: bad arguments");
  *domain = 0;
  int maxSteps = 0;
  for (int n = nDomains; n > 1; n >>= 1) ++maxSteps;  // floor(log2(nDomains))
  maxSteps += 1;
  int low = 0, up = nDomains - 1;
  if (offsetElem[low] < elemID && elemID <= offsetElem[low + 1]) {
    *domain = low;
  } else if (offsetElem[up] < elemID && elemID <= offsetElem[up + 1]) {
    *domain = up;
  } else {
    for (int i = 0; i < maxSteps; ++i) {
      const int mid = (up - low) / 2 + low;
      if (offsetElem[mid] < elemID && elemID <= offsetElem[mid + 1]) {
        *domain = mid;
        return SELFGPU_OK;
      } else if (elemID > offsetElem[mid + 1]) {
        low = mid + 1;
      } else {
        up = mid;
      }
    }
  }
  return SELFGPU_OK;
}

// Halo plan of one rank.  In: the global sideInfo (5,4,nElGlobal) and the
// decomposition.  Out: the rank's sideInfo (5,4,nLocal) with off-rank
// neighbours renumbered to halo elements nLocal+1.., the halo count, per peer
// the number of shared faces, and the concatenated (peer order) send and
// receive trace-block indices (block = side + 4 * local element, 0-based;
// a send block is one of this rank's sides, a receive block a halo side).
// sendBlocks and recvBlocks need room for 4 * nLocal entries.
int selfgpu_halo_plan(const int* sideInfoGlobal, int nElGlobal, int nDomains, const int* offsetElem, int rank,
                      int* sideInfoLocal, int* nHalo, int* peerCount, int* sendBlocks, int* recvBlocks) {
  if (!sideInfoGlobal || nElGlobal < 1 || nDomains < 1 || !offsetElem || rank < 0 || rank >= nDomains ||
      !sideInfoLocal || !nHalo || !peerCount || !sendBlocks || !recvBlocks)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_halo_plan: bad arguments");
  int rc = validate_side_info(sideInfoGlobal, nElGlobal, nElGlobal);
  if (rc != SELFGPU_OK) return rc;
  const int o = offsetElem[rank], nLocal = offsetElem[rank + 1] - offsetElem[rank];
  if (nLocal < 1) return set_error(SELFGPU_ERR_ARG, "selfgpu_halo_plan: empty rank");
  using Key = std::pair<long long, long long>;  // lower global (element, side) endpoint of a shared face
  struct Link {
    Key key;
    int send, recv;
  };
  std::vector<std::vector<Link>> links(nDomains);
  std::map<std::pair<int, int>, int> halo;  // (global element, side) -> halo index
  for (int e = 0; e < nLocal; ++e)
    for (int s = 0; s < 4; ++s) {
      const int* g = sideInfoGlobal + 5 * (s + 4 * (size_t)(o + e));
      int* l = sideInfoLocal + 5 * (s + 4 * (size_t)e);
      for (int k = 0; k < 5; ++k) l[k] = g[k];
      if (g[4] != 0) continue;
      const int e2g = g[2] - 1, s2 = g[3] / 10 - 1;
      if (e2g >= o && e2g < o + nLocal) {
        l[2] = e2g - o + 1;
        continue;
      }
      int peer = 0;
      selfgpu_elem_to_rank(nDomains, offsetElem, e2g + 1, &peer);
      if (peer == rank || e2g < offsetElem[peer] || e2g >= offsetElem[peer + 1])
        return set_error(SELFGPU_ERR_MESH, "selfgpu_halo_plan: neighbour rank lookup failed");
      auto it = halo.find({e2g, s2});
      const int h = it == halo.end() ? (int)halo.size() : it->second;
      if (it == halo.end()) halo[{e2g, s2}] = h;
      l[2] = nLocal + h + 1;
      const long long a = 4LL * (o + e) + s, b = 4LL * e2g + s2;
      links[peer].push_back({{std::min(a, b), std::max(a, b)}, s + 4 * e, s2 + 4 * (nLocal + h)});
    }
  int n = 0;
  for (int p = 0; p < nDomains; ++p) {
    std::sort(links[p].begin(), links[p].end(), [](const Link& x, const Link& y) { return x.key < y.key; });
    peerCount[p] = (int)links[p].size();
    for (const Link& k : links[p]) {
      sendBlocks[n] = k.send;
      recvBlocks[n] = k.recv;
      ++n;
    }
  }
  *nHalo = (int)halo.size();
  return SELFGPU_OK;
}

}  // extern "C"
