// autotune.cu — launch shapes of the post-filter stages and their cache.
//
// Every post-filter stage is a grid-stride launch over a flattened tile list,
// so its grid size (resident CTAs per SM) is free; superres also has a free
// tile width (output samples of a row per tile).  The shape in use comes from
// a per-process table keyed by (stage, 8-bit or high bit depth), seeded with
// defaults measured on B200 and overwritten by av1g_autotune_postfilter (api.cu),
// which times every candidate on a real batch.  The table can be saved to and
// loaded from a small text file ("stage hbd ctas_per_sm tile" per line), which
// av1g_engine_create loads when its config names one.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"

namespace av1g {

namespace {

std::mutex g_mu;
// What the autotuner picks on a 64 x 1080p batch on B200: grids several
// times the resident CTAs (deblock 6, CDEF and LR 4 per SM), so the tiles'
// uneven work evens out over many small CTAs instead of ending in a partial
// last wave.
StageShape g_shape[ST_COUNT][2] = {
    {{16, 0}, {16, 0}},    // deblock
    {{16, 0}, {16, 0}},    // CDEF
    {{16, 512}, {16, 512}},  // superres
    {{8, 0}, {8, 0}},      // loop restoration
    {{8, 0}, {8, 0}},      // film grain blend
};

}  // namespace

StageShape stage_shape(int stage, int hbd) {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_shape[stage][hbd ? 1 : 0];
}

void set_stage_shape(int stage, int hbd, const StageShape& sh) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_shape[stage][hbd ? 1 : 0] = sh;
}

int shape_grid(const StageShape& sh, int total) {
    const long long g = (long long)kSMs * (sh.ctas_per_sm > 0 ? sh.ctas_per_sm : 1);
    return (int)(total < g ? total : g);
}

bool shape_valid(int stage, const StageShape& sh) {
    if (sh.ctas_per_sm < 1 || sh.ctas_per_sm > 64) return false;
    if (stage == ST_SUPERRES) return sh.tile == 256 || sh.tile == 512 || sh.tile == 1024;
    return true;
}

av1g_status save_shapes(const char* path, std::string& err) {
    FILE* f = fopen(path, "w");
    if (!f) {
        err = std::string("cannot write ") + path;
        return AV1G_EINVAL;
    }
    fprintf(f, "# stage hbd ctas_per_sm tile  (stages: 0 deblock, 1 cdef, 2 superres, 3 lr, 4 film grain)\n");
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (int st = 0; st < ST_COUNT; st++)
            for (int h = 0; h < 2; h++) fprintf(f, "%d %d %d %d\n", st, h, g_shape[st][h].ctas_per_sm, g_shape[st][h].tile);
    }
    fclose(f);
    return AV1G_OK;
}

av1g_status load_shapes(const char* path, std::string& err) {
    FILE* f = fopen(path, "r");
    if (!f) {
        err = std::string("cannot read ") + path;
        return AV1G_EINVAL;
    }
    char line[256];
    int bad = 0;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        int st, h, c, t;
        if (sscanf(line, "%d %d %d %d", &st, &h, &c, &t) != 4 || st < 0 || st >= ST_COUNT || h < 0 || h > 1 ||
            !shape_valid(st, StageShape{c, t})) {
            bad++;
            continue;
        }
        set_stage_shape(st, h, StageShape{c, t});
    }
    fclose(f);
    if (bad) {
        err = std::string(path) + ": " + std::to_string(bad) + " malformed line(s) ignored";
        return AV1G_EINVAL;
    }
    return AV1G_OK;
}

}  // namespace av1g
