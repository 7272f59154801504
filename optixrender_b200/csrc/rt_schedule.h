// rt_schedule.h - the render server's wave planner, without CUDA.
//
// Given the admitted jobs that still have paths to issue (in admission
// order), the policy picks the group the next wave serves and then how many
// paths each of that group's jobs contributes, in at most `max_segments`
// segments of a wave of `capacity` path slots.  The server's groups are the
// plain jobs of scenes without media or textures (group 0), the plain jobs of
// scenes with them (group 1) and the guided jobs of scene k (group k + 2):
// one wave runs one build of the shade kernel and samples at most one guiding
// network, so a plain job's wave runs the same kernel as a Render() of it.
//   FIFO: the oldest job's group; jobs in admission order take all they can.
//   SRPT: the group of the job with the fewest paths left; jobs with the
//         fewest paths left first (ties by admission).
//   FAIR: groups in rotation; up to max_segments jobs taken round-robin split
//         the wave evenly, a job needing less than its share leaving the rest
//         to the others (water filling).
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <utility>
#include <vector>

namespace rti {

enum : int { kPlanFair = 0, kPlanFifo = 1, kPlanSrpt = 2 };

struct PlanJob {
    int64_t remaining;  // paths not yet issued (> 0)
    int group;          // jobs of one group may share a wave
};

struct PlanState {
    size_t rr = 0;       // round-robin position among the group's jobs (fair)
    size_t group_rr = 0; // rotation point over the groups (fair)
};

// Returns (index into `jobs`, paths) per segment; all segments share one group.
inline std::vector<std::pair<size_t, int64_t>> plan_wave(const std::vector<PlanJob>& jobs, int policy,
                                                         int64_t capacity, int max_segments, PlanState& st) {
    std::vector<std::pair<size_t, int64_t>> plan;
    if (jobs.empty() || capacity <= 0 || max_segments <= 0) return plan;
    int chosen = jobs.front().group;
    if (policy == kPlanSrpt) {
        size_t best = 0;
        for (size_t i = 1; i < jobs.size(); i++)
            if (jobs[i].remaining < jobs[best].remaining) best = i;
        chosen = jobs[best].group;
    } else if (policy == kPlanFair) {
        int best = -1, first = -1;
        for (const PlanJob& j : jobs) {
            if (first < 0 || j.group < first) first = j.group;
            if (j.group >= int(st.group_rr) && (best < 0 || j.group < best)) best = j.group;
        }
        chosen = best >= 0 ? best : first;
        st.group_rr = size_t(chosen) + 1;
    }
    std::vector<size_t> act;
    for (size_t i = 0; i < jobs.size(); i++)
        if (jobs[i].group == chosen) act.push_back(i);
    if (policy == kPlanFifo || policy == kPlanSrpt) {
        if (policy == kPlanSrpt)
            std::stable_sort(act.begin(), act.end(),
                             [&](size_t a, size_t b) { return jobs[a].remaining < jobs[b].remaining; });
        int64_t left = capacity;
        for (size_t i : act) {
            if (left == 0 || int(plan.size()) == max_segments) break;
            const int64_t take = std::min(jobs[i].remaining, left);
            plan.emplace_back(i, take);
            left -= take;
        }
        return plan;
    }
    const size_t k = std::min(act.size(), size_t(max_segments));
    const size_t start = st.rr % act.size();
    std::vector<size_t> pick;
    for (size_t n = 0; n < k; n++) pick.push_back(act[(start + n) % act.size()]);
    st.rr = start + k;
    std::vector<size_t> order(k);
    for (size_t n = 0; n < k; n++) order[n] = n;
    std::sort(order.begin(), order.end(),
              [&](size_t a, size_t b) { return jobs[pick[a]].remaining < jobs[pick[b]].remaining; });
    std::vector<int64_t> give(k, 0);
    int64_t left = capacity;
    for (size_t n = 0; n < k; n++) {
        const size_t i = order[n];
        give[i] = std::min(jobs[pick[i]].remaining, left / int64_t(k - n));
        left -= give[i];
    }
    for (size_t i = 0; i < k && left > 0; i++) {  // remainder of the integer split
        const int64_t extra = std::min(left, jobs[pick[i]].remaining - give[i]);
        give[i] += extra;
        left -= extra;
    }
    for (size_t i = 0; i < k; i++)
        if (give[i] > 0) plan.emplace_back(pick[i], give[i]);
    return plan;
}

}  // namespace rti
