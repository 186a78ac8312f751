// bx_amr_plan.cu -- the host side of dynamic AMR: BATL's refinement
// decisions (set_amr_criteria / regrid_batl of srcBATL, absent from the
// reference tree), restated from their documented behaviour
// (PARAM.XML:6658-6910: #AMRLEVELS, #AMR, #DOAMR, #AMRCRITERIA;
// Doc/Tex/grid.tex:50-110), and the remap table of bx_regrid.
//
//   * a block refines if ANY criterion exceeds its RefineLimit and its level
//     is below MaxBlockLevel;
//   * it coarsens if ALL criteria are below their CoarsenLimit, its level is
//     above MinBlockLevel and below MaxBlockLevel, all 2^nDim siblings are
//     leaves that may coarsen too, and no leaf next to their parent is finer
//     than they are (checked on the tree after the refinements);
//   * a refinement splits coarser neighbours (faces, edges, corners) until
//     neighbouring levels differ by at most one;
//   * refinements go in decreasing order of the largest criterion / limit
//     ratio, and the first one that would exceed MaxTotalBlocks ends them;
//   * the new blocks follow the Morton curve of the finest level.
//
// Host code only: bx_amr_plan runs without a device.
#include <algorithm>
#include <cstdint>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/bx200.h"
#include "bx_amr.h"
#include "bx_core.h"

namespace bx {
namespace {

// level (5 bits) and three 19-bit block indices
inline uint64_t pack(int lv, int i, int j, int k) {
  return ((uint64_t)lv << 57) | ((uint64_t)i << 38) | ((uint64_t)j << 19) | (uint64_t)k;
}
struct Key {
  int lv, c[3];
};
inline Key unpack(uint64_t q) {
  return Key{(int)(q >> 57), {(int)((q >> 38) & 0x7FFFF), (int)((q >> 19) & 0x7FFFF), (int)(q & 0x7FFFF)}};
}

uint64_t morton(uint32_t x, uint32_t y, uint32_t z) {
  uint64_t k = 0;
  for (int b = 0; b < 21; b++)
    k |= ((uint64_t)((x >> b) & 1) << (3 * b)) | ((uint64_t)((y >> b) & 1) << (3 * b + 1)) |
         ((uint64_t)((z >> b) & 1) << (3 * b + 2));
  return k;
}

struct Tree {
  int nDim;
  int nb0[3];
  bool per[3];
  std::unordered_set<uint64_t> leaves;
  std::vector<int> kids;    // octants a + 2b + 4c used by nDim
  std::vector<int> offs;    // neighbour offsets, (a+1) + 3 (b+1) + 9 (c+1)

  Tree(const bx_grid_desc *gd) {
    nDim = gd->nDim;
    for (int d = 0; d < 3; d++) {
      nb0[d] = d < nDim ? gd->nRootBlock[d] : 1;
      per[d] = gd->TypeBc[2 * d] == BX_BC_PERIODIC;
    }
    for (int o = 0; o < 8; o++)
      if ((nDim > 1 || !(o & 2)) && (nDim > 2 || !(o & 4))) kids.push_back(o);
    for (int c = -1; c <= 1; c++)
      for (int b = -1; b <= 1; b++)
        for (int a = -1; a <= 1; a++) {
          if ((a | b | c) == 0 || (nDim < 2 && b) || (nDim < 3 && c)) continue;
          offs.push_back((a + 1) + 3 * (b + 1) + 9 * (c + 1));
        }
    leaves.reserve(4 * (size_t)gd->nBlock);
    for (int b = 0; b < gd->nBlock; b++) {
      const int *q = gd->iLevelCoord_IB + 4 * b;
      leaves.insert(pack(q[0], q[1], q[2], q[3]));
    }
  }
  // level-lv block index c wrapped at periodic sides; false outside
  bool wrap(int lv, int c[3]) const {
    for (int d = 0; d < 3; d++) {
      const int n = d < nDim ? nb0[d] << lv : 1;
      if (c[d] < 0 || c[d] >= n) {
        if (d >= nDim || !per[d]) return false;
        c[d] = ((c[d] % n) + n) % n;
      }
    }
    return true;
  }
  // the leaf at level lv or coarser covering c; 0 (no key has all zero bits
  // except the root block at level 0, so use a flag) when none
  bool leaf_at(int lv, int c0[3], uint64_t &out) const {
    int c[3] = {c0[0], c0[1], c0[2]};
    if (!wrap(lv, c)) return false;
    for (int l2 = lv; l2 >= 0; l2--) {
      const int s = lv - l2;
      const uint64_t q = pack(l2, c[0] >> s, c[1] >> s, c[2] >> s);
      if (leaves.count(q)) { out = q; return true; }
    }
    return false;
  }
  void children(uint64_t q, uint64_t ch[8], int &n) const {
    const Key k = unpack(q);
    n = 0;
    for (int o : kids)
      ch[n++] = pack(k.lv + 1, 2 * k.c[0] + (o & 1), 2 * k.c[1] + ((o >> 1) & 1), 2 * k.c[2] + (o >> 2));
  }
  void split(uint64_t key, std::vector<uint64_t> &journal) {
    std::vector<uint64_t> work{key};
    while (!work.empty()) {
      const uint64_t q = work.back();
      work.pop_back();
      if (!leaves.erase(q)) continue;
      uint64_t ch[8];
      int n;
      children(q, ch, n);
      for (int m = 0; m < n; m++) leaves.insert(ch[m]);
      journal.push_back(q);
      for (int m = 0; m < n; m++) {
        const Key c = unpack(ch[m]);
        for (int o : offs) {
          int p[3] = {c.c[0] + o % 3 - 1, c.c[1] + (o / 3) % 3 - 1, c.c[2] + o / 9 - 1};
          uint64_t nk;
          if (leaf_at(c.lv, p, nk) && unpack(nk).lv < c.lv - 1) work.push_back(nk);
        }
      }
    }
  }
  void unsplit(const std::vector<uint64_t> &journal) {
    for (auto it = journal.rbegin(); it != journal.rend(); ++it) {
      uint64_t ch[8];
      int n;
      children(*it, ch, n);
      for (int m = 0; m < n; m++) leaves.erase(ch[m]);
      leaves.insert(*it);
    }
  }
  // is a leaf next to the region of parent finer than its children?
  bool finer_next_to(uint64_t parent) const {
    uint64_t ch[8];
    int n;
    children(parent, ch, n);
    const int lv = unpack(parent).lv + 1;
    for (int m = 0; m < n; m++) {
      const Key c = unpack(ch[m]);
      for (int o : offs) {
        int p[3] = {c.c[0] + o % 3 - 1, c.c[1] + (o / 3) % 3 - 1, c.c[2] + o / 9 - 1};
        int w[3] = {p[0], p[1], p[2]};
        if (!wrap(lv, w)) continue;
        const uint64_t q = pack(lv, w[0], w[1], w[2]);
        if (std::find(ch, ch + n, q) != ch + n) continue;
        uint64_t nk;
        if (!leaf_at(lv, p, nk)) return true;  // inside the domain and covered by finer leaves
      }
    }
    return false;
  }
};

}  // namespace

int amr_plan(const bx_grid_desc *gd, const bx_amr_params *p, const double *Crit_IB, std::vector<int> &lcNew,
             std::vector<int> &remap, bool &changed) {
  const int nB = gd->nBlock, nC = p->nCrit;
  std::vector<uint64_t> keys(nB);
  for (int b = 0; b < nB; b++) {
    const int *q = gd->iLevelCoord_IB + 4 * b;
    keys[b] = pack(q[0], q[1], q[2], q[3]);
  }
  std::vector<char> wantRef(nB), wantCoa(nB);
  std::vector<double> ratio(nB);
  for (int b = 0; b < nB; b++) {
    const int lv = gd->iLevelCoord_IB[4 * b];
    bool anyRef = false, allCoa = true;
    double r = -1e300;
    for (int q = 0; q < nC; q++) {
      const double c = Crit_IB[(size_t)b * nC + q];
      anyRef = anyRef || c > p->RefineLimit[q];
      allCoa = allCoa && c < p->CoarsenLimit[q];
      r = std::max(r, c / (p->RefineLimit[q] != 0.0 ? p->RefineLimit[q] : 1.0));
    }
    wantRef[b] = anyRef && lv < p->MaxBlockLevel;
    wantCoa[b] = allCoa && lv > p->MinBlockLevel && lv < p->MaxBlockLevel && !wantRef[b];
    ratio[b] = r;
  }
  // no block asks to refine or coarsen: the leaves stay, and when the old
  // list already follows the Morton order of the finest level (every list
  // this planner made does) the new grid is the old one, block for block
  if (std::none_of(wantRef.begin(), wantRef.end(), [](char w) { return w != 0; }) &&
      std::none_of(wantCoa.begin(), wantCoa.end(), [](char w) { return w != 0; })) {
    int mx = 0;
    for (int b = 0; b < nB; b++) mx = std::max(mx, gd->iLevelCoord_IB[4 * b]);
    bool inOrder = true;
    std::pair<uint64_t, int> prev{0, 0};
    for (int b = 0; b < nB && inOrder; b++) {
      const int *q = gd->iLevelCoord_IB + 4 * b;
      const int sh = mx - q[0];
      const std::pair<uint64_t, int> cur{morton((uint32_t)q[1] << sh, (uint32_t)q[2] << sh, (uint32_t)q[3] << sh),
                                         q[0]};
      inOrder = b == 0 || prev < cur;
      prev = cur;
    }
    if (inOrder) {
      lcNew.assign(gd->iLevelCoord_IB, gd->iLevelCoord_IB + 4 * (size_t)nB);
      remap.assign((size_t)kRemapInts * nB, 0);
      for (int b = 0; b < nB; b++) {
        remap[(size_t)kRemapInts * b] = kRemapCopy;
        remap[(size_t)kRemapInts * b + 1] = b + 1;
      }
      changed = false;
      return BX_OK;
    }
  }
  Tree t(gd);
  std::vector<int> cand;
  for (int b = 0; b < nB; b++)
    if (wantRef[b]) cand.push_back(b);
  std::stable_sort(cand.begin(), cand.end(), [&](int x, int y) {
    if (ratio[x] != ratio[y]) return ratio[x] > ratio[y];
    return x < y;
  });
  for (int b : cand) {
    if (!t.leaves.count(keys[b])) continue;
    std::vector<uint64_t> journal;
    t.split(keys[b], journal);
    if ((long)t.leaves.size() > p->MaxTotalBlocks) {
      t.unsplit(journal);
      break;
    }
  }
  // coarsening of whole sibling groups, decided on the refined tree
  std::unordered_map<uint64_t, int> groups;
  for (int b = 0; b < nB; b++) {
    if (!wantCoa[b] || !t.leaves.count(keys[b])) continue;
    const Key k = unpack(keys[b]);
    groups[pack(k.lv - 1, k.c[0] >> 1, k.c[1] >> 1, k.c[2] >> 1)]++;
  }
  std::vector<uint64_t> merge;
  for (const auto &gr : groups) {
    if (gr.second != (int)t.kids.size()) continue;
    uint64_t ch[8];
    int n;
    t.children(gr.first, ch, n);
    bool all = true;
    for (int m = 0; m < n && all; m++) all = t.leaves.count(ch[m]) > 0;
    if (all && !t.finer_next_to(gr.first)) merge.push_back(gr.first);
  }
  for (uint64_t q : merge) {
    uint64_t ch[8];
    int n;
    t.children(q, ch, n);
    for (int m = 0; m < n; m++) t.leaves.erase(ch[m]);
    t.leaves.insert(q);
  }
  // Morton order of the finest level
  std::vector<uint64_t> out(t.leaves.begin(), t.leaves.end());
  int mx = 0;
  for (uint64_t q : out) mx = std::max(mx, unpack(q).lv);
  std::vector<std::pair<uint64_t, int>> ord(out.size());
  for (size_t m = 0; m < out.size(); m++) {
    const Key k = unpack(out[m]);
    const int s = mx - k.lv;
    ord[m] = {morton((uint32_t)k.c[0] << s, (uint32_t)k.c[1] << s, (uint32_t)k.c[2] << s), k.lv};
  }
  std::vector<size_t> idx(out.size());
  for (size_t m = 0; m < idx.size(); m++) idx[m] = m;
  std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return ord[x] < ord[y]; });
  const int nNew = (int)out.size();
  lcNew.assign(4 * (size_t)nNew, 0);
  changed = nNew != nB;
  std::unordered_map<uint64_t, int> oldIndex;
  oldIndex.reserve(2 * (size_t)nB);
  for (int b = 0; b < nB; b++) oldIndex[keys[b]] = b;
  remap.assign((size_t)kRemapInts * nNew, 0);
  for (int b = 0; b < nNew; b++) {
    const uint64_t q = out[idx[b]];
    const Key k = unpack(q);
    lcNew[4 * b] = k.lv;
    for (int d = 0; d < 3; d++) lcNew[4 * b + 1 + d] = k.c[d];
    if (!changed && keys[b] != q) changed = true;
    int *R = remap.data() + (size_t)kRemapInts * b;
    auto it = oldIndex.find(q);
    if (it != oldIndex.end()) {
      R[0] = kRemapCopy;
      R[1] = it->second + 1;
      continue;
    }
    if (k.lv > 0 && (it = oldIndex.find(pack(k.lv - 1, k.c[0] >> 1, k.c[1] >> 1, k.c[2] >> 1))) != oldIndex.end()) {
      R[0] = kRemapProlong;
      R[1] = it->second + 1;
      R[2] = (k.c[0] & 1) + 2 * (k.c[1] & 1) + 4 * (k.c[2] & 1);
      continue;
    }
    R[0] = kRemapRestrict;
    for (int o = 0; o < 8; o++) {
      it = oldIndex.find(pack(k.lv + 1, 2 * k.c[0] + (o & 1), 2 * k.c[1] + ((o >> 1) & 1), 2 * k.c[2] + (o >> 2)));
      if (it == oldIndex.end()) return core_fail(BX_ERR_ARG, "new block %d changed by more than one level", b + 1);
      R[1 + o] = it->second + 1;
    }
  }
  return BX_OK;
}

}  // namespace bx

extern "C" int bx_amr_plan(const bx_grid_desc *gd, const bx_amr_params *p, const double *Crit_IB, int nBlockNewMax,
                           int *nBlockNew, int *iLevelCoordNew_IB, int *iRemap_IB, int *IsChanged) {
  if (!gd || !p || !Crit_IB || !nBlockNew || !gd->iLevelCoord_IB)
    return bx::core_fail(BX_ERR_ARG, "null argument");
  if (p->nCrit < 1 || p->nCrit > 3) return bx::core_fail(BX_ERR_ARG, "nCrit=%d (1..3)", p->nCrit);
  if (gd->nDim != 3) return bx::core_fail(BX_ERR_ARG, "dynamic AMR of 3D grids only");
  std::vector<int> lc, R;
  bool changed = false;
  int r = bx::amr_plan(gd, p, Crit_IB, lc, R, changed);
  if (r) return r;
  *nBlockNew = (int)(lc.size() / 4);
  if (IsChanged) *IsChanged = changed ? 1 : 0;
  if (*nBlockNew > nBlockNewMax)
    return bx::core_fail(BX_ERR_ARG, "the new grid has %d blocks, room for %d", *nBlockNew, nBlockNewMax);
  if (iLevelCoordNew_IB) std::copy(lc.begin(), lc.end(), iLevelCoordNew_IB);
  if (iRemap_IB) std::copy(R.begin(), R.end(), iRemap_IB);
  return BX_OK;
}
