// prr_main.cpp - the `prr` command: the reference's executable
// (prr.cpp:64-135 cmdinput, prr.cpp:345-404 main) over the C ABI.
//
//     prr -t <deck.params> [--device N] [--first F] [--count C]
//         [--batch B] [--out PREFIX]
//
// Renders every frame the deck defines and writes <out>image_<i>.png, as
// the reference does; the options after the deck are additions.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "prr.h"

static void show_usage(const char *name)
{
    fprintf(stderr,
            "Usage: %s <option(s)>\n"
            "Options:\n"
            "\t-t, --trace\t\tStart the ray tracing with the given file as parameters\n"
            "\t-h, --help\t\tShow this help message\n"
            "\t--device N\t\tCUDA device (default 0)\n"
            "\t--first F, --count C\tRender frames [F, F+C) (default: all)\n"
            "\t--batch B\t\tFrames per render call (default 16)\n"
            "\t--out PREFIX\t\tOutput prefix (default: the deck's tracer.out)\n\n",
            name);
}

int main(int argc, char **argv)
{
    std::string deck, out;
    bool have_out = false;
    int device = 0, first = 0, count = -1, batch = 16;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&](const char *what) -> const char * {
            if (i + 1 >= argc) {
                fprintf(stderr, "ERROR::: %s requires one argument.\n\n", what);
                exit(2);
            }
            return argv[++i];
        };
        if (a == "-h" || a == "--help") { show_usage(argv[0]); return 0; }
        else if (a == "-t" || a == "--trace") deck = next("-t and --trace");
        else if (a == "--device") device = atoi(next("--device"));
        else if (a == "--first") first = atoi(next("--first"));
        else if (a == "--count") count = atoi(next("--count"));
        else if (a == "--batch") batch = atoi(next("--batch"));
        else if (a == "--out") { out = next("--out"); have_out = true; }
        else { show_usage(argv[0]); return 2; }
    }
    if (deck.empty()) {
        fprintf(stderr, "ERROR::: No .params file was given. You need to specify a problem file when running PRR "
                        "(e.g. prr -t input/sim.params).\n\n");
        return 2;
    }
    prr_ctx *ctx = nullptr;
    prr_status s = prr_create(device, &ctx);
    if (s != PRR_OK) {
        fprintf(stderr, "prr: cannot create a context on device %d: %s\n", device, prr_status_string(s));
        return 1;
    }
    prr_stats st;
    s = prr_run_deck(ctx, deck.c_str(), first, count, have_out ? out.c_str() : nullptr, batch, &st);
    if (s != PRR_OK) {
        fprintf(stderr, "prr: %s: %s\n", prr_status_string(s), prr_last_error(ctx));
        prr_destroy(ctx);
        return 1;
    }
    printf("prr: %lld rays, %lld RKF/Euler attempts, %.1f ms on the device (%.2f Mrays/s)\n", (long long)st.rays,
           (long long)st.attempts, st.kernel_ms, st.kernel_ms > 0 ? st.rays / (st.kernel_ms * 1e3) : 0.0);
    prr_destroy(ctx);
    return 0;
}
