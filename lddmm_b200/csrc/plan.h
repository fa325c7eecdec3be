// Host-side work plans of the persistent time-loop sweeps (persist.cuh): which CTA
// takes which (row group, j range) segments, and for the cluster form which CTA
// finalises each row group shared by several CTAs of a cluster.  Plain C++ (no device
// code), built once per context.
#pragma once

#include <algorithm>
#include <vector>

#include "layout.h"

namespace lddmm {

constexpr int kPlanSub = 32;          // j entries per staged sub-tile (kSub)
constexpr int kPlanMaxJobParts = 8;   // parts of a row group in the cluster form (kMaxJobParts)

// Work plan of the persistent sweeps: the step's work (row groups x their j ranges,
// laid end to end in unit order) cut into G contiguous shares, one per CTA.  Cuts
// inside a row group are rounded to the 32-entry sub-tile and moved to the row group's
// edge when they would leave a part shorter than kMinPart entries.  With little work
// per CTA (under kSplitMin entries) row groups are not cut at all: each CTA takes whole
// row groups and G is at most the row-group count.
struct HostPlan {
  std::vector<int4> segs;       // (unit, j begin, j end, part) in CTA order
  std::vector<int> cta_seg;     // G + 1 offsets into segs
  std::vector<int2> unit_parts; // (parts, first partial slot)
  int slots = 0;
};

constexpr long long kMinPart = 32;
constexpr long long kSplitMin = 512;

inline HostPlan plan_sweeps(const std::vector<int2> &units, const std::vector<PairDesc> &hpd,
                            int G_max) {
  const int nu = (int)units.size();
  std::vector<long long> us(nu + 1, 0);
  for (int u = 0; u < nu; ++u) us[u + 1] = us[u] + hpd[units[u].x].Npad;
  const long long W = us[nu];
  const bool cut = W / std::max(G_max, 1) >= kSplitMin;
  const int G = cut ? G_max : std::max(1, std::min(G_max, nu));
  std::vector<long long> b(G + 1, 0);
  b[G] = W;
  for (int k = 1; k < G; ++k) {
    long long x;
    if (cut) {
      const long long w = W * k / G;
      int u = (int)(std::upper_bound(us.begin(), us.end(), w) - us.begin()) - 1;
      u = std::min(std::max(u, 0), nu - 1);
      const long long J = us[u + 1] - us[u];
      long long off = (w - us[u] + kPlanSub / 2) / kPlanSub * kPlanSub;
      if (off < kMinPart) off = 0;
      else if (J - off < kMinPart) off = J;
      x = us[u] + off;
    } else {
      x = us[(long long)nu * k / G];
    }
    b[k] = std::max(b[k - 1], std::min(x, W));
  }
  HostPlan h;
  h.cta_seg.assign(G + 1, 0);
  h.unit_parts.assign(nu, make_int2(0, 0));
  std::vector<int> parts(nu, 0);
  int u0 = 0;
  for (int k = 0; k < G; ++k) {
    h.cta_seg[k] = (int)h.segs.size();
    while (u0 < nu && us[u0 + 1] <= b[k]) ++u0;
    for (int v = u0; v < nu && us[v] < b[k + 1]; ++v) {
      const long long lo = std::max(b[k], us[v]) - us[v];
      const long long hi = std::min(b[k + 1], us[v + 1]) - us[v];
      if (hi > lo) h.segs.push_back(make_int4(v, (int)lo, (int)hi, parts[v]++));
    }
  }
  h.cta_seg[G] = (int)h.segs.size();
  for (int v = 0; v < nu; ++v) {
    h.unit_parts[v] = make_int2(parts[v], h.slots);
    if (parts[v] > 1) h.slots += parts[v];
  }
  return h;
}

// Work plan of the cluster-form persistent sweeps: the row groups split into ncl
// contiguous ranges of whole row groups, one per cluster, minimising the largest
// range's work (binary search on the bound, greedy fill); each cluster's entries cut
// into C CTA shares as in plan_sweeps.  Only a CTA's first and last segment can be part
// of a row group shared with other CTAs (slots 0 and 1); the CTA holding a shared row
// group's first part finalises it (at most one per CTA: only a CTA's last segment can
// be a first part).  CTA k * C + r is rank r of cluster k.  max_share: the largest CTA
// share in entries.
struct ClusterHostPlan {
  std::vector<int4> segs;       // (unit, j begin, j end, kind: 0 whole, 1 / 2 slot 0 / 1)
  std::vector<int> cta_seg;     // ncl * C + 1 offsets into segs
  std::vector<int2> job;        // per CTA: (unit, parts) or (-1, 0)
  std::vector<int> job_src;     // per CTA x kPlanMaxJobParts: rank << 1 | slot
  long long max_share = 0;
  bool ok = false;
};

inline ClusterHostPlan plan_cluster_sweeps(const std::vector<int2> &units,
                                           const std::vector<PairDesc> &hpd, int C, int ncl) {
  ClusterHostPlan h;
  const int nu = (int)units.size();
  if (nu == 0 || C < 1 || C > kPlanMaxJobParts || ncl < 1) return h;
  std::vector<long long> w(nu);
  long long tot = 0, wmax = 0;
  for (int u = 0; u < nu; ++u) {
    w[u] = hpd[units[u].x].Npad;
    tot += w[u];
    wmax = std::max(wmax, w[u]);
  }
  auto ranges = [&](long long cap) {
    int g = 1;
    long long acc = 0;
    for (int u = 0; u < nu; ++u) {
      if (acc + w[u] > cap) {
        ++g;
        acc = 0;
      }
      acc += w[u];
    }
    return g;
  };
  long long lo = wmax, hi = tot;
  while (lo < hi) {
    const long long mid = (lo + hi) / 2;
    if (ranges(mid) <= ncl) hi = mid;
    else lo = mid + 1;
  }
  std::vector<int> ub(1, 0);  // unit range of each cluster
  {
    long long acc = 0;
    for (int u = 0; u < nu; ++u) {
      if (acc + w[u] > lo) {
        ub.push_back(u);
        acc = 0;
      }
      acc += w[u];
    }
    while ((int)ub.size() < ncl + 1) ub.push_back(nu);
  }
  const int G = ncl * C;
  h.cta_seg.assign(G + 1, 0);
  h.job.assign(G, make_int2(-1, 0));
  h.job_src.assign((size_t)G * kPlanMaxJobParts, 0);
  for (int k = 0; k < ncl; ++k) {
    const int u0 = ub[k], u1 = ub[k + 1];
    std::vector<long long> us(1, 0);
    for (int u = u0; u < u1; ++u) us.push_back(us.back() + w[u]);
    const long long L = us.back();
    std::vector<long long> b(C + 1, 0);
    b[C] = L;
    for (int r = 1; r < C; ++r) {
      const long long x = L * r / C;
      int v = (int)(std::upper_bound(us.begin(), us.end(), x) - us.begin()) - 1;
      v = std::min(std::max(v, 0), std::max(u1 - u0 - 1, 0));
      long long off = 0;
      if (u1 > u0) {
        const long long J = us[v + 1] - us[v];
        off = (x - us[v] + kPlanSub / 2) / kPlanSub * kPlanSub;
        if (off < kMinPart) off = 0;
        else if (J - off < kMinPart) off = J;
      }
      b[r] = std::max(b[r - 1], std::min(us[v] + off, L));
    }
    std::vector<std::vector<int2>> parts(u1 - u0);  // (rank, slot) per shared row group
    for (int r = 0; r < C; ++r) {
      const int cta = k * C + r;
      h.cta_seg[cta] = (int)h.segs.size();
      h.max_share = std::max(h.max_share, b[r + 1] - b[r]);
      const int first = (int)h.segs.size();
      for (int v = 0; v < u1 - u0; ++v) {
        const long long lo2 = std::max(b[r], us[v]) - us[v];
        const long long hi2 = std::min(b[r + 1], us[v + 1]) - us[v];
        if (hi2 > lo2) h.segs.push_back(make_int4(u0 + v, (int)lo2, (int)hi2, 0));
      }
      const int last = (int)h.segs.size() - 1;
      for (int q = first; q <= last; ++q) {
        int4 &sg = h.segs[q];
        if (sg.y == 0 && sg.z == (int)w[sg.x]) continue;  // a whole row group
        if (q != first && q != last) return h;  // cannot happen: middle segments are whole
        const int slot = (q == first) ? 0 : 1;
        sg.w = 1 + slot;
        parts[sg.x - u0].push_back(make_int2(r, slot));
      }
    }
    for (int v = 0; v < u1 - u0; ++v) {
      const std::vector<int2> &pv = parts[v];
      if (pv.empty()) continue;
      if ((int)pv.size() > kPlanMaxJobParts) return h;
      const int cta = k * C + pv[0].x;
      if (h.job[cta].x >= 0) return h;  // one job per CTA
      h.job[cta] = make_int2(u0 + v, (int)pv.size());
      for (size_t q = 0; q < pv.size(); ++q)
        h.job_src[(size_t)cta * kPlanMaxJobParts + q] = (pv[q].x << 1) | pv[q].y;
    }
  }
  h.cta_seg[G] = (int)h.segs.size();
  h.ok = true;
  return h;
}

}  // namespace lddmm
