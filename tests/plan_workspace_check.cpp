/* Test driver for tests/test_plan_workspace_cpu.py: compiles the ghost fill
 * of each mesh named on the command line twice, without and with a
 * compiler workspace that is reused (and given the previous plan's arrays)
 * from one mesh to the next, as fx_amr_adapt does, and prints whether the
 * two plans are identical byte for byte.  Each mesh is a pair of files
 * <prefix>.cfg (an fx_config) and <prefix>.desc (fx_block_desc entries). */
#include "../fornaxamr_b200/csrc/fx_plan.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

bool load(const std::string &prefix, fx_config &cfg, std::vector<fx_block_desc> &d)
{
    FILE *f = fopen((prefix + ".cfg").c_str(), "rb");
    if (!f) return false;
    const bool ok = fread(&cfg, sizeof cfg, 1, f) == 1;
    fclose(f);
    if (!ok) return false;
    f = fopen((prefix + ".desc").c_str(), "rb");
    if (!f) return false;
    fx_block_desc x;
    d.clear();
    while (fread(&x, sizeof x, 1, f) == 1) d.push_back(x);
    fclose(f);
    return !d.empty();
}

template <class T>
bool same_vec(const std::vector<T> &a, const std::vector<T> &b)
{
    return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(T)) == 0);
}

bool same_plan(const FxPlan &a, const FxPlan &b)
{
    const FxProgram &g = a.ghost, &h = b.ghost;
    return same_vec(g.cell_ops, h.cell_ops) && same_vec(g.face_ops, h.face_ops) && same_vec(g.p_ops, h.p_ops) &&
        same_vec(g.b_ops, h.b_ops) && same_vec(g.cell_begin, h.cell_begin) && same_vec(g.face_begin, h.face_begin) &&
        same_vec(g.p_begin, h.p_begin) && same_vec(g.b_begin, h.b_begin) && same_vec(a.active, b.active) &&
        same_vec(a.flux_corr, b.flux_corr) && same_vec(a.flux_corr_begin, b.flux_corr_begin) &&
        same_vec(a.emf_corr, b.emf_corr) && same_vec(a.emf_corr_begin, b.emf_corr_begin) &&
        a.stats.emitted_cell_ops == b.stats.emitted_cell_ops && a.stats.emitted_face_ops == b.stats.emitted_face_ops &&
        a.stats.rewired == b.stats.rewired && a.stats.dead == b.stats.dead;
}

} // namespace

int main(int argc, char **argv)
{
    FxPlanWorkspace *ws = fx_plan_workspace_new();
    FxPlan current;
    int bad = 0;
    for (int i = 1; i < argc; ++i) {
        fx_config cfg;
        std::vector<fx_block_desc> d;
        if (!load(argv[i], cfg, d)) {
            printf("%s unreadable\n", argv[i]);
            return 2;
        }
        FxPlan fresh, reused;
        std::string e1, e2;
        const bool o1 = fx_build_plan(cfg, (int)d.size(), d.data(), fresh, &e1);
        const bool o2 = fx_build_plan(cfg, (int)d.size(), d.data(), reused, &e2, ws);
        const bool same = o1 && o2 && same_plan(fresh, reused) && !fresh.ghost.cell_ops.empty();
        printf("%s %s\n", argv[i], same ? "same" : "DIFFERENT");
        bad += same ? 0 : 1;
        FxPlan old = std::move(current);
        current = std::move(reused);
        fx_plan_workspace_recycle(ws, std::move(old));
    }
    fx_plan_workspace_free(ws);
    return bad;
}
