// plan_check.cu -- host-only check of the batched split planner
// (batch_plan / batch_max_split in starlab_b200/csrc/kernels.h), built and
// run by tests/test_split_plan.py without a GPU.
//
// The batched kernels write split partials to part[split * ni + i]; the
// ensemble sizes its buffer per cluster as n * batch_max_split(nj_pad,
// min_tiles) and every task reads j in [split * jper, split * jper + jper)
// of the padded j-set.  For every layout, lane shape, tasks-wanted setting
// and fewest-tiles setting, over i- and j-counts from 1 to 2^18, this
// checks that a plan stays inside those bounds and covers the j-set exactly:
//   jper a positive multiple of the tile; every split non-empty; the splits
//   cover all nj_pad j; nsplit <= batch_max_split; n_tasks = i-tiles x
//   nsplit with the i-tiles covering ni; H a power of two dividing the warps.
// The mixed mode's FP64 refinement pass (refine.cu) plans its flagged
// particles the same way with refine_tasks_wanted; its partials buffer holds
// refine_partial_records(ni) records, checked against nsplit x flagged.
// Prints "ok <plans checked>" or the first violation, and exits 1 on one.
#include <cstdio>
#include <vector>
#include "kernels.h"

using namespace g6;

// The batched launches' base shape (batch_config in force.cu): 32 i-lanes,
// one i per thread, 8 warps; H and the split settings vary below.
static ForceConfig base_config() {
    ForceConfig c;
    c.il = 32;
    c.r = 1;
    c.warps = 8;
    c.H = 4;
    c.nsplit = 0;
    return c;
}

static int fail(const char *what, int kmode, const ForceConfig &c, int ni, int nj_pad, const ForceParams &p) {
    std::printf("FAIL %s: kmode=%d nsplit_cfg=%d min_tiles=%d H_cfg=%d ni=%d nj_pad=%d -> jper=%d nsplit=%d H=%d\n",
                what, kmode, c.nsplit, c.min_tiles, c.H, ni, nj_pad, p.jper, p.nsplit, p.H);
    return 1;
}

int main() {
    std::vector<int> sizes;
    for (int v = 1; v <= (1 << 18); v = v < 8 ? v + 1 : v + v / 3) sizes.push_back(v);
    for (int v : {255, 256, 257, 511, 512, 513, 1023, 1024, 1025, 16384, 16385, 65536, 262144}) sizes.push_back(v);
    const int kmodes[3] = {kKernF64, kKernMixedDS, kKernMixedP};
    const int nsplits[5] = {0, 1, 296, 592, 1184};
    const int min_tiles[4] = {1, 2, 4, 8};
    const int hs[4] = {1, 2, 4, 8};
    long long checked = 0;
    for (int kmode : kmodes) {
        const int T = tile_of(kmode);
        for (int h : hs)
            for (int ns : nsplits)
                for (int mt : min_tiles) {
                    ForceConfig c = base_config();
                    c.H = h;
                    c.nsplit = ns;
                    c.min_tiles = mt;
                    for (int nj : sizes) {
                        const int nj_pad = (nj + T - 1) / T * T;
                        const int ntiles = nj_pad / T;
                        const int max_split = batch_max_split(kmode, nj_pad, mt);
                        for (int ni : sizes) {
                            if (ni > nj) continue;  // a block never holds more i than the cluster
                            ForceParams p{};
                            p.ni = ni;
                            p.nj = nj;
                            p.nj_pad = nj_pad;
                            int nt = -1;
                            batch_plan(kmode, c, p, nt);
                            ++checked;
                            if (p.jper < T || p.jper % T != 0) return fail("jper not a positive multiple of the tile", kmode, c, ni, nj_pad, p);
                            if (p.nsplit < 1) return fail("no split", kmode, c, ni, nj_pad, p);
                            if ((long long)p.nsplit * p.jper < nj_pad) return fail("splits do not cover the j-set", kmode, c, ni, nj_pad, p);
                            if ((long long)(p.nsplit - 1) * p.jper >= nj_pad) return fail("empty split", kmode, c, ni, nj_pad, p);
                            if (p.nsplit > max_split) return fail("nsplit above batch_max_split", kmode, c, ni, nj_pad, p);
                            if (p.nsplit > ntiles) return fail("more splits than tiles", kmode, c, ni, nj_pad, p);
                            if (p.H < 1 || c.warps % p.H != 0 || (p.H & (p.H - 1)) != 0) return fail("bad H", kmode, c, ni, nj_pad, p);
                            const int itile = batch_item_itile(kmode, c, ni);
                            if (itile < 1) return fail("empty i-tile", kmode, c, ni, nj_pad, p);
                            const long long n_itiles = (ni + itile - 1) / itile;
                            if (nt != n_itiles * p.nsplit) return fail("task count", kmode, c, ni, nj_pad, p);
                            if (n_itiles * itile < ni) return fail("i-tiles do not cover ni", kmode, c, ni, nj_pad, p);
                        }
                    }
                }
    }
    // the refinement's FP64 pass: `count` flagged i of a call, any j-count
    for (int nj : sizes) {
        const int nj_pad = (nj + tile_of(kKernF64) - 1) / tile_of(kKernF64) * tile_of(kKernF64);
        for (int count : sizes) {
            ForceConfig c = base_config();
            c.nsplit = refine_tasks_wanted(count, nj_pad);
            ForceParams p{};
            p.ni = count;
            p.nj = nj;
            p.nj_pad = nj_pad;
            int nt = -1;
            batch_plan(kKernF64, c, p, nt);
            ++checked;
            if ((size_t)p.nsplit * (size_t)count > refine_partial_records(count))
                return fail("refinement partials above refine_partial_records", kKernF64, c, count, nj_pad, p);
            if ((long long)p.nsplit * p.jper < nj_pad || (long long)(p.nsplit - 1) * p.jper >= nj_pad)
                return fail("refinement splits do not tile the j-set", kKernF64, c, count, nj_pad, p);
        }
    }
    std::printf("ok %lld\n", checked);
    return 0;
}
