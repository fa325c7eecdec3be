"""Host-side work plans of the persistent time-loop sweeps (lddmm_b200/csrc/plan.h),
compiled here with the host compiler and checked on batches of even and uneven pairs
for every cluster size: every (row group, j) entry is covered exactly once, a row
group of the cluster form never crosses a cluster, a CTA's split segments sit in its
first and last slot, each shared row group has exactly one finalising CTA whose part
list names the parts in CTA order, and the L2 form's parts count matches."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

HARNESS = r'''
#include <cstdio>
#include <vector>
#include <algorithm>
#include <vector_types.h>
#include <vector_functions.h>
#include "plan.h"
using namespace lddmm;

static int check_cluster(const std::vector<int> &npad, int C, int ncl) {
  std::vector<PairDesc> hpd(npad.size());
  std::vector<int2> units;
  for (size_t p = 0; p < npad.size(); ++p) {
    hpd[p].Npad = npad[p];
    for (int g = 0; g < npad[p] / 16; ++g) units.push_back(make_int2((int)p, g));
  }
  ClusterHostPlan h = plan_cluster_sweeps(units, hpd, C, ncl);
  if (!h.ok) return 1;
  const int G = C * ncl, nu = (int)units.size();
  std::vector<std::vector<std::pair<int, int>>> cover(nu), parts(nu);
  for (int k = 0; k < G; ++k) {
    const int first = h.cta_seg[k], last = h.cta_seg[k + 1] - 1;
    for (int q = first; q <= last; ++q) {
      const int4 s = h.segs[q];
      const int J = npad[units[s.x].x];
      if (s.y < 0 || s.z > J || s.y >= s.z) return 2;
      cover[s.x].push_back({s.y, s.z});
      const bool whole = s.y == 0 && s.z == J;
      if (whole != (s.w == 0)) return 3;
      if (s.w == 1 && q != first) return 4;
      if (s.w == 2 && (q != last || q == first)) return 5;
      if (s.w) parts[s.x].push_back({k, s.w - 1});
    }
  }
  for (int u = 0; u < nu; ++u) {
    std::sort(cover[u].begin(), cover[u].end());
    int x = 0;
    for (auto &c : cover[u]) {
      if (c.first != x) return 6;
      x = c.second;
    }
    if (x != npad[units[u].x]) return 7;
    if (parts[u].empty()) continue;
    const int cl = parts[u][0].first / C;
    for (auto &pp : parts[u])
      if (pp.first / C != cl) return 8;
    const int cta = parts[u][0].first;
    if (h.job[cta].x != u || h.job[cta].y != (int)parts[u].size()) return 9;
    for (int q = 0; q < h.job[cta].y; ++q) {
      const int src = h.job_src[cta * kPlanMaxJobParts + q];
      if ((src >> 1) != parts[u][q].first % C || (src & 1) != parts[u][q].second) return 10;
    }
  }
  int jobs = 0;
  for (auto &j : h.job) jobs += j.x >= 0;
  int shared = 0;
  for (int u = 0; u < nu; ++u) shared += !parts[u].empty();
  return jobs == shared ? 0 : 11;
}

static int check_l2(const std::vector<int> &npad, int G) {
  std::vector<PairDesc> hpd(npad.size());
  std::vector<int2> units;
  for (size_t p = 0; p < npad.size(); ++p) {
    hpd[p].Npad = npad[p];
    for (int g = 0; g < npad[p] / 16; ++g) units.push_back(make_int2((int)p, g));
  }
  HostPlan h = plan_sweeps(units, hpd, G);
  std::vector<int> n(units.size(), 0);
  std::vector<long long> len(units.size(), 0);
  for (const int4 &s : h.segs) {
    n[s.x]++;
    len[s.x] += s.z - s.y;
  }
  for (size_t u = 0; u < units.size(); ++u)
    if (len[u] != npad[units[u].x] || n[u] != h.unit_parts[u].x) return 20;
  return 0;
}

int main() {
  std::vector<std::vector<int>> cases = {{2624}, std::vector<int>(8, 2624), {64, 128, 64}};
  std::vector<int> mix;
  unsigned s = 1;
  for (int i = 0; i < 40; ++i) {
    s = s * 1103515245u + 12345u;
    mix.push_back(64 * (1 + (int)((s >> 16) % 40)));
  }
  cases.push_back(mix);
  for (auto &cs : cases) {
    for (int C = 1; C <= kPlanMaxJobParts; ++C)
      for (int ncl : {296 / C, 200 / C + 1, 3}) {
        const int rc = check_cluster(cs, C, ncl);
        if (rc) {
          printf("cluster plan C=%d ncl=%d failed: %d\n", C, ncl, rc);
          return rc;
        }
      }
    for (int G : {296, 148, 7}) {
      const int rc = check_l2(cs, G);
      if (rc) {
        printf("L2 plan G=%d failed: %d\n", G, rc);
        return rc;
      }
    }
  }
  printf("ok\n");
  return 0;
}
'''


def _cuda_include():
    for base in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if base and os.path.exists(os.path.join(base, "include", "vector_types.h")):
            return os.path.join(base, "include")
    return None


@pytest.mark.skipif(shutil.which("g++") is None or _cuda_include() is None,
                    reason="needs g++ and the CUDA headers")
def test_persistent_work_plans(tmp_path):
    src = tmp_path / "plan_check.cpp"
    exe = tmp_path / "plan_check"
    src.write_text(HARNESS)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "lddmm_b200", "csrc"),
                    "-I", _cuda_include(), str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
