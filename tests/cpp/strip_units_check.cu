// Host-side checks of rgbd-flow_b200/csrc/pipeline.cuh.  The strip SOR's work units: for ragged
// steps, every band layout (the fixed band heights and the balancing model's layouts) must cut each
// item's strips into bands that start on a multiple of 32 rows, cover the strip's rows exactly
// once, and the work list must hold every (item, strip, band) once, largest band first.  The
// register whole-level SOR kernels' padded half-row pitch and cluster shapes (check_level_pitch).
// Runs on the host only (no kernel is launched).  Prints one line per case and exits non-zero on
// the first violation.
#include <cstdio>
#include <cstdlib>
#include <set>
#include <tuple>

#include "../../rgbd-flow_b200/csrc/pipeline.cuh"

using namespace rgbdflow;

struct Item {
    int W, H;
};

static int fail(const char* what, int a, int b)
{
    std::printf("FAIL %s (%d, %d)\n", what, a, b);
    return 1;
}

static int check(const char* name, const std::vector<Item>& items, int seg, bool balanced)
{
    std::vector<int> which;
    for (int i = 0; i < (int)items.size(); i++) which.push_back(i);
    HostParams hp{};
    hp.strip_seg = seg;
    BandMap lay;
    if (balanced) lay = strip_balanced_bands(items, which, seg > 0 ? seg : 128, 148);
    for (const auto& e : lay) {
        int tot = 0;
        for (int h : e.second) {
            if (h <= 0 || h > 256) return fail("band height", e.first, h);
            tot += h;
        }
        if (tot != e.first) return fail("layout does not cover the strip", e.first, tot);
    }
    const std::vector<StripUnit> u = strip_units(items, which, hp, 148, balanced ? &lay : nullptr);
    std::set<std::tuple<int, int, int>> rows;  // (item, strip x0, row)
    int prev_h = 1 << 30;
    for (const auto& x : u) {
        const Item& it = items[x.item];
        if (x.x0 % kStripW != 0 || x.x0 < 0 || x.x0 >= it.W) return fail("strip column", x.item, x.x0);
        if (x.ya % 32 != 0 || x.ya < 0 || x.yb > it.H || x.yb <= x.ya) return fail("band rows", x.ya, x.yb);
        const int h = x.yb - x.ya;
        if (h > prev_h) return fail("units not largest first", prev_h, h);
        prev_h = h;
        for (int r = x.ya; r < x.yb; r++)
            if (!rows.insert(std::make_tuple(x.item, x.x0, r)).second) return fail("row covered twice", x.item, r);
    }
    size_t want = 0;
    for (const auto& it : items) want += (size_t)((it.W + kStripW - 1) / kStripW) * it.H;
    if (rows.size() != want) return fail("rows not covered", (int)rows.size(), (int)want);
    std::printf("ok %s seg %d%s: %zu units", name, seg, balanced ? " balanced" : "", u.size());
    for (const auto& e : lay) {
        std::printf(" H%d:", e.first);
        for (size_t q = 0; q < e.second.size(); q++) std::printf("%s%d", q ? "/" : "", e.second[q]);
    }
    std::printf("\n");
    return 0;
}

// The padded half-row pitch of the register whole-level kernels: at least a zero position each
// side, 2 x pitch = row length (mod 32), at most 15 positions of padding; and the cluster shapes the
// plan picks for them fit the 64 KB of shared memory those kernels are given.
static int check_level_pitch()
{
    for (int hwp = 4; hwp <= 512; hwp += 4) {
        const int rp = level_reg_rp(hwp);
        if (rp < hwp + 2 || ((2 * rp - hwp) & 31) != 0 || rp - (hwp + 2) > 15) return fail("pitch", hwp, rp);
    }
    HostParams hp{};
    hp.sor_level = 1;
    hp.level_reg = 1;
    int shapes = 0;
    for (int H = 8; H <= 400; H += 7)
        for (int hwp = 4; hwp <= 200; hwp += 4) {
            const auto sh = level_cluster_reg_shape(hp, H, hwp);
            if (sh.first == 0) continue;
            shapes++;
            const int B = (H + sh.first - 1) / sh.first;
            if (level_cluster_reg_smem_bytes<float>(B, hwp) > 64 * 1024) return fail("cluster smem", H, hwp);
            if (B * (sh.first - 1) >= H) return fail("empty cluster rank", H, sh.first);
        }
    std::printf("ok level pitch: %d cluster shapes\n", shapes);
    return 0;
}

int main()
{
    if (check_level_pitch()) return 1;
    std::vector<std::pair<const char*, std::vector<Item>>> cases;
    cases.push_back({"16 x 640x480", std::vector<Item>(16, Item{640, 480})});
    cases.push_back({"16 x 320x240", std::vector<Item>(16, Item{320, 240})});
    cases.push_back({"1 x 640x480", std::vector<Item>(1, Item{640, 480})});
    {
        std::vector<Item> mix;
        for (int i = 0; i < 24; i++) mix.push_back({160, 120});
        for (int i = 0; i < 24; i++) mix.push_back({320, 240});
        for (int i = 0; i < 16; i++) mix.push_back({640, 480});
        cases.push_back({"64-pair mix", mix});
    }
    cases.push_back({"ragged", {{333, 217}, {640, 480}, {129, 64}, {1000, 97}, {200, 300}}});
    for (const auto& c : cases)
        for (int seg : {0, 32, 64, 96, 128, 192, 256})
            for (int bal = 0; bal <= 1; bal++)
                if (check(c.first, c.second, seg, bal != 0)) return 1;
    return 0;
}
