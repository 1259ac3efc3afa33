// frame_loop.cpp - the deck-driven frame loop: main() of the reference
// (prr.cpp:345-404) and the per-frame renderframe (prr.cpp:237-341) over the
// C ABI.  Textures named by the deck are read once (tracer.bimage1 as the
// sky, sphereN.tex per sphere), frames are rendered in batches (the
// persistent scheduler fills the GPU across frames) and each frame is
// written as <out>image_<i>.png, the reference's file name (prr.cpp:336).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "prr.h"
#include "prr_internal.h"

namespace {

prr_status fail(prr_ctx *ctx, prr_status s, const std::string &msg)
{
    ctx->err = msg;
    return s;
}

std::string deck_str(const prr_deck *d, const char *block, const char *key)
{
    size_t n = prr_deck_get(d, block, key, nullptr, 0);
    std::string v(n, '\0');
    if (n) prr_deck_get(d, block, key, &v[0], n + 1);
    return v;
}

prr_status upload_file(prr_ctx *ctx, int id, const std::string &path)
{
    uint8_t *px = nullptr;
    int w = 0, h = 0;
    char err[512] = {0};
    prr_status s = prr_image_load(path.c_str(), &px, &w, &h, err, sizeof(err));
    if (s != PRR_OK) return fail(ctx, s, std::string("texture: ") + err);
    s = prr_upload_texture(ctx, id, px, w, h);
    prr_image_free(px);
    return s;
}

}  // namespace

extern "C" prr_status prr_run_deck(prr_ctx *ctx, const char *path, int first, int count, const char *out_prefix,
                                   int batch, prr_stats *stats)
{
    if (!ctx) return PRR_ERR_INVALID;
    if (!path) return fail(ctx, PRR_ERR_INVALID, "prr_run_deck: null deck path");
    char err[512] = {0};
    prr_deck *deck = nullptr;
    prr_status s = prr_deck_load(path, &deck, err, sizeof(err));
    if (s != PRR_OK) return fail(ctx, s, err);
    struct Guard {
        prr_deck *d;
        ~Guard() { prr_deck_free(d); }
    } guard{deck};
    const int nframes = prr_deck_frame_count(deck);
    if (nframes == 0) return fail(ctx, PRR_ERR_INVALID, "there are no frames to be rendered in the deck (prr.cpp:214-218)");
    if (first < 0 || first >= nframes) return fail(ctx, PRR_ERR_INVALID, "first frame out of range");
    const int last = count < 0 ? nframes : std::min(nframes, first + count);
    if (batch < 1) batch = 16;
    // textures, once (prr.cpp:360-365 and the Sphere constructor, scene/sphere.h:23)
    std::string sky = deck_str(deck, "tracer", "bimage1");
    if (!sky.empty() && (s = upload_file(ctx, 0, sky)) != PRR_OK) return s;
    prr_frame_desc f0;
    if ((s = prr_deck_frame(deck, first, &f0, err, sizeof(err))) != PRR_OK) return fail(ctx, s, err);
    for (int k = 0; k < f0.nspheres; k++) {
        if (f0.spheres[k].texture_id < 0) continue;
        bool seen = false;
        for (int j = 0; j < k; j++) seen |= f0.spheres[j].texture_id == f0.spheres[k].texture_id;
        if (seen) continue;
        std::string t = deck_str(deck, ("sphere" + std::to_string(k)).c_str(), "tex");
        if ((s = upload_file(ctx, f0.spheres[k].texture_id, t)) != PRR_OK) return s;
    }
    // a metric plug-in named by the deck (spacetime.metric = <library>.so) replaces main/metric.h's header
    int plugin_metric = -1;
    if (f0.metric == PRR_METRIC_PLUGIN0) {
        const std::string lib = deck_str(deck, "spacetime", "metric");
        if ((s = prr_load_metric_plugin(ctx, lib.c_str(), &plugin_metric)) != PRR_OK) return s;
    }
    std::string prefix = out_prefix ? std::string(out_prefix) : deck_str(deck, "tracer", "out");
    prr_stats total;
    memset(&total, 0, sizeof(total));
    std::vector<prr_frame_desc> descs;
    std::vector<uint8_t> rgb;
    for (int f = first; f < last; f += batch) {
        const int nb = std::min(batch, last - f);
        descs.resize(nb);
        size_t npx = 0;
        for (int k = 0; k < nb; k++) {
            if ((s = prr_deck_frame(deck, f + k, &descs[k], err, sizeof(err))) != PRR_OK) return fail(ctx, s, err);
            if (plugin_metric >= 0) descs[k].metric = plugin_metric;
            npx += (size_t)descs[k].width * (size_t)std::max(descs[k].height, 0);
        }
        rgb.resize(npx * 3);
        prr_stats st;
        if ((s = prr_render(ctx, descs.data(), nb, rgb.data(), nullptr, &st)) != PRR_OK) return s;
        size_t off = 0;
        for (int k = 0; k < nb; k++) {
            const prr_frame_desc &d = descs[k];
            std::string file = prefix + "image_" + std::to_string(f + k) + ".png";
            if (prr_png_write(file.c_str(), rgb.data() + off, d.width, d.height) != PRR_OK)
                return fail(ctx, PRR_ERR_IO, "cannot write " + file);
            off += (size_t)d.width * d.height * 3;
        }
        total.rays += st.rays; total.attempts += st.attempts; total.accepted += st.accepted;
        total.n_escaped += st.n_escaped; total.n_captured += st.n_captured; total.n_intersection += st.n_intersection;
        total.n_infinite += st.n_infinite; total.n_math_error += st.n_math_error; total.n_fp64 += st.n_fp64;
        total.kernel_ms += st.kernel_ms; total.trace_ms += st.trace_ms; total.kernel_launches += st.kernel_launches;
    }
    if (stats) *stats = total;
    return PRR_OK;
}
