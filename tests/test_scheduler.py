"""The render server's wave planner (optixrender_b200/csrc/rt_schedule.h),
compiled for the host: which group of jobs a wave serves and how many paths
each job contributes, under the FIFO, SRPT and fair policies."""
import subprocess

import numpy as np
import pytest

from conftest import ROOT

FAIR, FIFO, SRPT = 0, 1, 2

DRIVER = r"""
#include <cstdio>
#include "rt_schedule.h"
// stdin: policy capacity max_segments calls n, then n lines "remaining group";
// the same jobs are planned `calls` times (state carried), each plan printed
// as one line of "index:paths" pairs.
int main() {
    int policy, maxseg, calls, n;
    long long cap;
    while (std::scanf("%d %lld %d %d %d", &policy, &cap, &maxseg, &calls, &n) == 5) {
        std::vector<rti::PlanJob> jobs(n);
        for (auto& j : jobs) {
            long long r;
            std::scanf("%lld %d", &r, &j.group);
            j.remaining = r;
        }
        rti::PlanState st;
        for (int c = 0; c < calls; c++) {
            for (auto& p : rti::plan_wave(jobs, policy, cap, maxseg, st)) std::printf("%zu:%lld ", p.first, (long long)p.second);
            std::printf("\n");
        }
        std::printf("--\n");
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def planner(tmp_path_factory):
    d = tmp_path_factory.mktemp("sched")
    (d / "drv.cpp").write_text(DRIVER)
    exe = d / "drv"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "optixrender_b200" / "csrc"), str(d / "drv.cpp"),
                    "-o", str(exe)], check=True)

    def run(cases):
        text = ""
        for policy, cap, maxseg, calls, jobs in cases:
            text += f"{policy} {cap} {maxseg} {calls} {len(jobs)}\n" + "".join(f"{r} {g}\n" for r, g in jobs)
        out = subprocess.run([str(exe)], input=text, capture_output=True, text=True, check=True).stdout
        res, cur = [], []
        for line in out.splitlines():
            if line == "--":
                res.append(cur)
                cur = []
            else:
                cur.append([(int(a), int(b)) for a, b in (t.split(":") for t in line.split())])
        return res

    return run


def test_fifo_and_srpt_order(planner):
    jobs = [(500, 0), (100, 0), (300, 0)]
    fifo, srpt = planner([(FIFO, 700, 16, 1, jobs), (SRPT, 700, 16, 1, jobs)])
    assert fifo[0] == [(0, 500), (1, 100), (2, 100)]  # admission order
    assert srpt[0] == [(1, 100), (2, 300), (0, 300)]  # fewest paths left first
    (seg,) = planner([(FIFO, 10_000, 2, 1, jobs)])
    assert seg[0] == [(0, 500), (1, 100)]  # at most max_segments jobs per wave


def test_fair_water_filling_and_rotation(planner):
    (plans,) = planner([(FAIR, 900, 16, 1, [(100, 0), (1000, 0), (1000, 0)])])
    assert sorted(plans[0]) == [(0, 100), (1, 400), (2, 400)]  # the small job's unused share goes to the others
    (plans,) = planner([(FAIR, 100, 2, 3, [(1000, 0)] * 3)])
    firsts = [sorted(i for i, _ in p) for p in plans]
    assert firsts == [[0, 1], [0, 2], [1, 2]]  # two jobs per wave, taken round-robin
    assert all(sum(n for _, n in p) == 100 for p in plans)


def test_groups(planner):
    # job 0 plain, job 1 guided on scene 0 (group 1), job 2 guided on scene 1 (group 2)
    jobs = [(900, 0), (50, 1), (300, 2)]
    fifo, srpt, fair = planner([(FIFO, 1000, 16, 1, jobs), (SRPT, 1000, 16, 1, jobs), (FAIR, 1000, 16, 4, jobs)])
    assert fifo[0] == [(0, 900)]  # the oldest job's group only
    assert srpt[0] == [(1, 50)]   # the smallest job's group
    assert [p[0][0] for p in fair] == [0, 1, 2, 0]  # groups in rotation


def test_random_invariants(planner):
    rng = np.random.default_rng(5)
    cases = []
    for _ in range(300):
        n = int(rng.integers(1, 40))
        jobs = [(int(rng.integers(1, 5000)), int(rng.integers(0, 3))) for _ in range(n)]
        cases.append((int(rng.integers(0, 3)), int(rng.integers(1, 20000)), int(rng.integers(1, 17)), 3, jobs))
    for (policy, cap, maxseg, _, jobs), plans in zip(cases, planner(cases)):
        for p in plans:
            assert p, "a wave is planned whenever a job has work"
            idx = [i for i, _ in p]
            assert len(set(idx)) == len(idx) and len(p) <= maxseg
            assert len({jobs[i][1] for i in idx}) == 1  # one group per wave
            assert all(0 < take <= jobs[i][0] for i, take in p)
            total = sum(take for _, take in p)
            assert total <= cap
            group = jobs[idx[0]][1]
            members = [i for i, (_, g) in enumerate(jobs) if g == group]
            rem = [jobs[i][0] for i in members]
            if policy == FIFO:  # admission order
                assert total == min(cap, sum(rem[:maxseg]))
            elif policy == SRPT:  # fewest paths left first
                assert total == min(cap, sum(sorted(rem)[:maxseg]))
            else:  # work-conserving over the jobs chosen for the wave
                assert len(p) == min(len(members), maxseg) or total == cap
                assert total == cap or all(take == jobs[i][0] for i, take in p)
