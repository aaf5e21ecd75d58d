// Host-side coverage check of the sweeps' task plans in
// mhd_gpu_acc_b200/csrc/sweep.cuh (built and run by test_plans.py; no GPU).
// For grid extents from 1 cell to beyond the benchmark's 4096 and every work
// size the launches and the batch autotuner use, the tasks of x_plan (row
// segments) and y_plan (row bands of a column strip), enumerated through
// plan_task exactly as the kernels do, must cover every (row or strip, cell)
// pair exactly once, each task at least one cell long and inside the extent,
// and plan_task must report no task at or past plan_tasks.  Prints the first
// failure and exits 1.
#include <cstdio>
#include <vector>

#include "sweep.cuh"

using namespace mhd;

static int failures = 0;

static void fail(const char* what, int total, int size, long long k) {
    if (failures++ < 10) std::printf("FAIL %s: extent %d, work size %d, task %lld\n", what, total, size, k);
}

static void check(const SweepPlan& pl, int total, int width, int size) {
    for (int p = 0; p < 3; ++p)
        if (pl.len[p] < 1 || pl.n[p] < 0) fail("phase length / count", total, size, -1);
    if (pl.lo[0] != 0 || pl.lo[3] != total || pl.lo[1] > pl.lo[2] || pl.lo[2] > total)
        fail("phase bounds", total, size, -1);
    std::vector<unsigned char> hit((size_t)total * width, 0);
    const long long n = plan_tasks(pl, width);
    for (long long k = 0; k < n; ++k) {
        int idx = -1, start = -1, len = -1;
        if (!plan_task(pl, k, width, idx, start, len)) {
            fail("task missing", total, size, k);
            continue;
        }
        if (idx < 0 || idx >= width || start < 0 || len < 1 || start + len > total) {
            fail("task out of range", total, size, k);
            continue;
        }
        for (int c = start; c < start + len; ++c) hit[(size_t)idx * total + c] += 1;
    }
    for (long long k = n; k < n + 2 * width + 2; ++k) {
        int idx, start, len;
        if (plan_task(pl, k, width, idx, start, len)) fail("task past the end", total, size, k);
    }
    for (size_t i = 0; i < hit.size(); ++i)
        if (hit[i] != 1) {
            fail(hit[i] ? "cell covered twice" : "cell not covered", total, size, (long long)i);
            break;
        }
}

int main() {
    std::vector<int> extents;
    for (int t = 1; t <= 300; ++t) extents.push_back(t);
    for (int t : {316, 320, 508, 511, 512, 513, 668, 800, 1019, 1020, 1021, 1024, 2044, 2047, 2048, 2049, 3000,
                  4032, 4095, 4096, 4097, 5000})
        extents.push_back(t);
    long long plans = 0;
    for (int total : extents) {
        // x: segments of 4 * xrpw chunks (launch shapes and batch autotuner candidates)
        for (int xrpw : {1, 2, 3, 4, 6, 8, 12, 16, 24}) {
            check(x_plan(total, 4 * xrpw), total, 3, xrpw);
            if (x_plan(total, 4 * xrpw).len[0] != x_seg_len(4 * xrpw)) fail("x segment length", total, xrpw, -1);
            ++plans;
        }
        // y: bands of `per` rows over the strips
        for (int per : {1, 2, 4, 7, 14, 16, 20, 24, 28, 32, 48, 56, 64, 80, 128}) {
            check(y_plan(total, per), total, 3, per);
            ++plans;
        }
    }
    std::printf("%lld plans checked, %d failures\n", plans, failures);
    return failures ? 1 : 0;
}
