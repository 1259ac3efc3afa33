// deck.cpp - the reference's input decks, read with the reference's rules,
// and the deck-driven frame loop.
//
//   readParams         main/io.h:21-58         -> parse_file()
//   par/pari/parf      main/Parameters.cpp:20-44 -> prr_deck_get/geti/getf
//   headerExists/parExists                     -> prr_deck_has_block/has
//   checkFrame         prr.cpp:139-153         -> prr_deck_frame_count
//   createScene, setupScene, updateScene, renderframe's frame set-up
//                      prr.cpp:159-198,245-253; main/Spacetime.cpp:17-44
//                                              -> prr_deck_frame
//   main's frame loop and image.save           prr.cpp:345-404, 336
//                                              -> prr_run_deck
//
// Deck keys the reference does not have (all optional; defaults reproduce
// the reference): spacetime.metric (flat | schwarzschild | kerr | the path of
// a metric plug-in library; default schwarzschild, the header main/metric.h:12
// selects), tracer.mode
// (reference | physical), tracer.precision (fp32 | fp64 | split),
// camera.model (spherical | pinhole | panorama), camera.seed (random /
// jittered SSAA),
// tracer.rtol / tracer.atol (default eps), tracer.maxsteps (10000),
// tracer.horizon (stop at r <= r_+ + horizon; default 0.001 as
// metrics/schwarzschild.cuh:70), tracer.fxaa (0/1), tracer.bgfilter
// (rms2x2 | bilinear).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "prr.h"

typedef std::map<std::string, std::map<std::string, std::string>> Map2d;

struct prr_deck {
    Map2d p;
    int nspheres = 0;
};

namespace {

void put_err(char *buf, size_t len, const std::string &msg)
{
    if (!buf || !len) return;
    size_t n = std::min(len - 1, msg.size());
    memcpy(buf, msg.data(), n);
    buf[n] = 0;
}

// substr with the reference's unsigned (32-bit) index arithmetic: positions
// found by std::string::find are stored in `unsigned`, so "not found"
// becomes 0xFFFFFFFF, first + 1 wraps to 0 and the count wraps to "rest of
// the string".  The reference relies on these wraps for lines without '<',
// '>' or '=' (main/io.h:31-49).
std::string sub32(const std::string &s, unsigned pos, unsigned count)
{
    if (pos > s.size()) throw std::out_of_range("substr");
    return s.substr(pos, count);
}

std::string between(const std::string &s, char open, char close)
{
    unsigned first = (unsigned)s.find(open);
    unsigned last = (unsigned)s.find(close);
    return sub32(s, first + 1u, last - first - 1u);
}

// readParams (main/io.h:21-58) over one stream.
void parse_stream(std::istream &input, Map2d &params)
{
    std::string block;
    for (std::string line; std::getline(input, line);) {
        bool has_us = line.find('_') != std::string::npos, has_lt = line.find('<') != std::string::npos;
        if (!has_us && !has_lt) continue;  // no parameter and no block name
        try {
            if (has_us) {  // any '_' makes the line a block header
                unsigned first = (unsigned)line.find('_');
                unsigned last = (unsigned)line.find_last_of('_');
                block = sub32(line, first + 1u, last - first - 1u);
                continue;
            }
            size_t eq = line.find('=');
            std::string left = line.substr(0, eq);
            std::string right = line.substr(eq + 1, line.length() - 1);  // eq == npos: the whole line
            std::string key, val;
            if (!left.empty()) key = between(left, '<', '>');
            if (!right.empty()) val = between(right, '<', '>');
            params[block][key] = val;
        } catch (const std::out_of_range &) {
            // the reference would terminate on this line; keep going
        }
    }
}

bool parse_file(const std::string &fname, Map2d &params)
{
    std::ifstream input(fname);
    if (!input.good()) return false;
    parse_stream(input, params);
    return true;
}

void count_spheres(prr_deck *d)
{
    d->nspheres = 0;
    for (int i = 0; i < 10000; i++)  // Spacetime::setupScene (main/Spacetime.cpp:17-20)
        if (!d->p.count("sphere" + std::to_string(i))) { d->nspheres = i; break; }
}

bool has_block(const prr_deck *d, const std::string &h) { return d->p.count(h) != 0; }

bool has_key(const prr_deck *d, const std::string &h, const std::string &k)
{
    auto it = d->p.find(h);
    return it != d->p.end() && it->second.count(k) != 0;
}

std::string par(const prr_deck *d, const std::string &h, const std::string &k)
{
    return has_key(d, h, k) ? d->p.at(h).at(k) : std::string();
}

int pari(const prr_deck *d, const std::string &h, const std::string &k)
{
    if (!has_key(d, h, k)) return 0;
    try { return std::stoi(d->p.at(h).at(k)); } catch (const std::exception &) { return 0; }
}

float parf(const prr_deck *d, const std::string &h, const std::string &k, float dflt = 0.0f)
{
    if (!has_key(d, h, k)) return dflt;
    try { return std::stof(d->p.at(h).at(k)); } catch (const std::exception &) { return dflt; }
}

// deg * M_PI / 180.0f evaluated in double and stored as float, as
// prr.cpp:195,246-247 do.
float deg2rad(float deg) { return (float)(deg * M_PI / 180.0f); }

}  // namespace

extern "C" {

prr_status prr_deck_load(const char *path, prr_deck **out, char *errbuf, size_t errlen)
{
    if (!path || !out) { put_err(errbuf, errlen, "prr_deck_load: null argument"); return PRR_ERR_INVALID; }
    *out = nullptr;
    prr_deck *d = new prr_deck();
    // cmdinput (prr.cpp:125-131) refuses a main deck it cannot open
    if (!parse_file(path, d->p)) { put_err(errbuf, errlen, std::string("cannot open deck ") + path); delete d; return PRR_ERR_IO; }
    // init(), prr.cpp:208-210: the trajectory and scene decks named by the
    // tracer block are read into the same table (paths relative to the
    // working directory; a file that cannot be opened adds nothing, as in
    // the reference).
    for (const char *k : {"traj", "scene"}) {
        std::string sub = par(d, "tracer", k);
        if (!sub.empty()) parse_file(sub, d->p);
    }
    count_spheres(d);
    *out = d;
    return PRR_OK;
}

prr_status prr_deck_parse_string(const char *text, prr_deck **out)
{
    if (!text || !out) return PRR_ERR_INVALID;
    prr_deck *d = new prr_deck();
    std::istringstream in{std::string(text)};
    parse_stream(in, d->p);
    count_spheres(d);
    *out = d;
    return PRR_OK;
}

void prr_deck_free(prr_deck *d) { delete d; }

int prr_deck_has_block(const prr_deck *d, const char *block) { return d && block && has_block(d, block) ? 1 : 0; }

int prr_deck_has(const prr_deck *d, const char *block, const char *key)
{
    return d && block && key && has_key(d, block, key) ? 1 : 0;
}

size_t prr_deck_get(const prr_deck *d, const char *block, const char *key, char *buf, size_t len)
{
    if (!d || !block || !key) return 0;
    std::string v = par(d, block, key);
    if (buf && len) {
        size_t n = std::min(len - 1, v.size());
        memcpy(buf, v.data(), n);
        buf[n] = 0;
    }
    return v.size();
}

int prr_deck_geti(const prr_deck *d, const char *block, const char *key)
{
    return d && block && key ? pari(d, block, key) : 0;
}

float prr_deck_getf(const prr_deck *d, const char *block, const char *key, float dflt)
{
    return d && block && key ? parf(d, block, key, dflt) : dflt;
}

int prr_deck_frame_count(const prr_deck *d)
{
    if (!d) return 0;
    for (int i = 0; i < 100000; i++) {
        std::string h = "frame" + std::to_string(i);
        if (!(has_key(d, h, "x") && has_key(d, h, "y") && has_key(d, h, "z") && has_key(d, h, "a") && has_key(d, h, "b")))
            return i;
    }
    return 0;
}

int prr_deck_sphere_count(const prr_deck *d) { return d ? d->nspheres : 0; }

size_t prr_deck_sphere_texture(const prr_deck *d, int sphere, char *buf, size_t len)
{
    if (!d || sphere < 0 || sphere >= d->nspheres) return 0;
    return prr_deck_get(d, ("sphere" + std::to_string(sphere)).c_str(), "tex", buf, len);
}

prr_status prr_deck_frame(const prr_deck *d, int frame, prr_frame_desc *out, char *errbuf, size_t errlen)
{
    if (!d || !out) { put_err(errbuf, errlen, "prr_deck_frame: null argument"); return PRR_ERR_INVALID; }
    const int nframes = prr_deck_frame_count(d);
    if (frame < 0 || frame >= nframes) {
        put_err(errbuf, errlen, "frame " + std::to_string(frame) + " is not fully specified (x, y, z, a, b); the deck has " +
                                    std::to_string(nframes) + " frames");
        return PRR_ERR_INVALID;
    }
    if (d->nspheres > PRR_MAX_SPHERES) {
        put_err(errbuf, errlen, "the scene has " + std::to_string(d->nspheres) + " spheres; at most " +
                                    std::to_string(PRR_MAX_SPHERES) + " are supported");
        return PRR_ERR_UNSUPPORTED;
    }
    prr_frame_desc f;
    prr_frame_desc_defaults(&f);
    // ---- spacetime (createScene, prr.cpp:162-181) ----
    const bool bh = pari(d, "spacetime", "hasBlackHole") == 1;
    float mass = bh ? parf(d, "spacetime", "mass") : 0.0f;
    f.spin = bh ? parf(d, "spacetime", "spin") : 0.0f;
    std::string metric = par(d, "spacetime", "metric");
    if (!bh) f.metric = PRR_METRIC_FLAT;
    else if (metric.empty() || metric == "schwarzschild") f.metric = PRR_METRIC_SCHWARZSCHILD;
    else if (metric == "kerr") f.metric = PRR_METRIC_KERR;
    else if (metric == "flat") f.metric = PRR_METRIC_FLAT;
    else if (metric.size() > 3 && metric.compare(metric.size() - 3, 3, ".so") == 0)
        f.metric = PRR_METRIC_PLUGIN0;  // a metric plug-in library: prr_run_deck loads it and sets the id
    else { put_err(errbuf, errlen, "unknown spacetime metric '" + metric + "' (flat, schwarzschild, kerr, or a plug-in .so)"); return PRR_ERR_INVALID; }
    // ---- plasma emission (the plasma fields main/Spacetime.h:50-51 declares;
    //      keys of this library, PHYSICAL mode, prr_emission_desc) ----
    std::string emis = par(d, "spacetime", "emission");
    if (emis.empty() || emis == "none") f.emission = PRR_EMISSION_NONE;
    else if (emis == "disk") f.emission = PRR_EMISSION_DISK;
    else if (emis == "grid") {
        put_err(errbuf, errlen, "grid emission takes its plasma from prr_upload_plasma, not from a deck");
        return PRR_ERR_UNSUPPORTED;
    } else { put_err(errbuf, errlen, "unknown spacetime emission '" + emis + "' (none, disk)"); return PRR_ERR_INVALID; }
    f.emis.index = parf(d, "spacetime", "emisIndex", f.emis.index);
    f.emis.height = parf(d, "spacetime", "emisHeight", f.emis.height);
    f.emis.r_in = parf(d, "spacetime", "emisRin", f.emis.r_in);
    f.emis.r_out = parf(d, "spacetime", "emisRout", f.emis.r_out);
    f.emis.spectral_index = parf(d, "spacetime", "emisAlpha", f.emis.spectral_index);
    f.emis.absorb = parf(d, "spacetime", "emisAbsorb", f.emis.absorb);
    f.emis.gain = parf(d, "spacetime", "emisGain", f.emis.gain);
    if (has_key(d, "spacetime", "emisSense")) f.emis.sense = pari(d, "spacetime", "emisSense");
    std::string cmap = par(d, "spacetime", "emisMap");
    if (cmap.empty() || cmap == "afmhot") f.emis.colormap = PRR_CMAP_AFMHOT;
    else if (cmap == "grey") f.emis.colormap = PRR_CMAP_GREY;
    else { put_err(errbuf, errlen, "unknown emission colour map '" + cmap + "' (afmhot, grey)"); return PRR_ERR_INVALID; }
    // ---- tracer (prr.cpp:184-190) ----
    std::string solver = par(d, "tracer", "solver");
    if (solver == "euler") f.solver = PRR_SOLVER_EULER;
    else if (solver == "rkf") f.solver = PRR_SOLVER_RKF45;
    else if (solver == "rk" || solver == "adams" || solver == "gragg" || solver == "dormand" || solver == "taylor") {
        // known to Parameters::getSolver but without an integrator
        // (renderframe launches no tracing kernel for them, prr.cpp:295-305)
        put_err(errbuf, errlen, "solver '" + solver + "' has no integrator (euler and rkf do)");
        return PRR_ERR_UNSUPPORTED;
    } else f.solver = PRR_SOLVER_EULER;  // Parameters::getSolver's fallback (main/Parameters.h:18-22)
    f.hmin = parf(d, "tracer", "hmin");
    f.hmax = parf(d, "tracer", "hmax");
    f.h = parf(d, "tracer", "h");
    f.eps = parf(d, "tracer", "eps");
    f.rout = parf(d, "tracer", "rout1");
    std::string mode = par(d, "tracer", "mode");
    if (mode.empty() || mode == "reference") f.mode = PRR_MODE_REFERENCE;
    else if (mode == "physical") f.mode = PRR_MODE_PHYSICAL;
    else { put_err(errbuf, errlen, "unknown tracer mode '" + mode + "' (reference, physical)"); return PRR_ERR_INVALID; }
    std::string prec = par(d, "tracer", "precision");
    if (prec.empty() || prec == "fp32") f.precision = PRR_PREC_FP32;
    else if (prec == "fp64") f.precision = PRR_PREC_FP64;
    else if (prec == "split") f.precision = PRR_PREC_SPLIT;
    else { put_err(errbuf, errlen, "unknown tracer precision '" + prec + "' (fp32, fp64, split)"); return PRR_ERR_INVALID; }
    f.rtol = parf(d, "tracer", "rtol", f.eps);
    f.atol = parf(d, "tracer", "atol", f.eps);
    if (has_key(d, "tracer", "maxsteps")) f.max_steps = pari(d, "tracer", "maxsteps");
    f.horizon_eps = parf(d, "tracer", "horizon", 0.001f);
    f.fxaa = pari(d, "tracer", "fxaa") ? 1 : 0;
    std::string bgf = par(d, "tracer", "bgfilter");
    f.bg_filter = bgf == "bilinear" ? PRR_BG_BILINEAR : PRR_BG_RMS2X2;
    f.background_id = par(d, "tracer", "bimage1").empty() ? -1 : 0;
    // ---- camera (prr.cpp:194-195) ----
    std::string ssaa = par(d, "camera", "SSAA");
    if (ssaa == "none") f.ssaa = PRR_SSAA_NONE;
    else if (ssaa == "regular") f.ssaa = PRR_SSAA_REGULAR;
    else if (ssaa == "random") f.ssaa = PRR_SSAA_RANDOM;      // PHYSICAL mode (the reference never launches its kernel)
    else if (ssaa == "jittered") f.ssaa = PRR_SSAA_JITTERED;  // likewise
    else if (ssaa == "poisson" || ssaa == "rotated") {
        put_err(errbuf, errlen, "SSAA distribution '" + ssaa + "' has no implementation (none in the reference either)");
        return PRR_ERR_UNSUPPORTED;
    } else f.ssaa = PRR_SSAA_REGULAR;  // Parameters::getSSAA's fallback (main/Parameters.h:24-29)
    f.ssaa_seed = (uint32_t)pari(d, "camera", "seed");
    std::string model = par(d, "camera", "model");
    if (model.empty() || model == "spherical") f.camera = PRR_CAMERA_SPHERICAL;
    else if (model == "pinhole") f.camera = PRR_CAMERA_PINHOLE;
    else if (model == "panorama") f.camera = PRR_CAMERA_PANORAMA;
    else { put_err(errbuf, errlen, "unknown camera model '" + model + "' (spherical, pinhole, panorama)"); return PRR_ERR_INVALID; }
    f.samples = pari(d, "camera", "SSAAsamples");
    f.vfov = deg2rad(parf(d, "camera", "vfov"));
    f.width = pari(d, "camera", "width");
    f.height = pari(d, "camera", "height");
    // ---- spheres: setupScene then updateScene(k) for k = 0..frame; each
    //      update keeps the previous value of a key the deck lacks
    //      (main/Spacetime.cpp:17-44).  The mass override of renderframe
    //      (prr.cpp:253) also carries over from frame to frame. ----
    std::vector<float> c(3 * d->nspheres), r(d->nspheres);
    for (int s = 0; s < d->nspheres; s++) {
        std::string hd = "sphere" + std::to_string(s);
        c[3 * s] = parf(d, hd, "x0"); c[3 * s + 1] = parf(d, hd, "y0"); c[3 * s + 2] = parf(d, hd, "z0");
        r[s] = parf(d, hd, "r0");
    }
    std::map<std::string, int> tex_ids;
    for (int k = 0; k <= frame; k++) {
        std::string fs = std::to_string(k);
        for (int s = 0; s < d->nspheres; s++) {
            std::string hd = "sphere" + std::to_string(s);
            c[3 * s] = parf(d, hd, "x" + fs, c[3 * s]);
            c[3 * s + 1] = parf(d, hd, "y" + fs, c[3 * s + 1]);
            c[3 * s + 2] = parf(d, hd, "z" + fs, c[3 * s + 2]);
            r[s] = parf(d, hd, "r" + fs, r[s]);
        }
        mass = parf(d, "frame" + fs, "mass", mass);
    }
    f.mass = mass;
    if (f.metric == PRR_METRIC_FLAT) f.mass = bh ? mass : 0.0f;
    f.nspheres = d->nspheres;
    int next_id = 1;
    for (int s = 0; s < d->nspheres; s++) {
        prr_sphere &S = f.spheres[s];
        S.center[0] = c[3 * s]; S.center[1] = c[3 * s + 1]; S.center[2] = c[3 * s + 2];
        S.radius = r[s];
        std::string tex = par(d, "sphere" + std::to_string(s), "tex");
        if (tex.empty()) { S.texture_id = -1; continue; }
        auto it = tex_ids.find(tex);
        if (it == tex_ids.end()) it = tex_ids.emplace(tex, next_id++).first;
        S.texture_id = it->second;
    }
    // ---- camera pose of this frame (prr.cpp:245-247) ----
    std::string h = "frame" + std::to_string(frame);
    f.cam_pos[0] = parf(d, h, "x"); f.cam_pos[1] = parf(d, h, "y"); f.cam_pos[2] = parf(d, h, "z");
    f.cam_alpha = deg2rad(parf(d, h, "a"));
    f.cam_beta = deg2rad(parf(d, h, "b"));
    *out = f;
    return PRR_OK;
}

}  // extern "C"
