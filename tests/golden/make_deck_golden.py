"""Generates tests/golden/decks.json from the REFERENCE ITSELF: each deck
below is parsed by the reference's own readParams (main/io.h:21-58) and read
back through its own getters par/pari/parf/headerExists/parExists
(main/Parameters.cpp:10-44) and checkFrame (prr.cpp:139-153), all compiled
for the host in oracle/_ref by oracle/ref/build_ref.sh.

    python tests/golden/make_deck_golden.py

The decks are written here to exercise the parse rules and their quirks:
comments, CRLF line ends, values with '_' (which open a block), lines
without '=', '<' or '>', empty and bare-underscore headers, std::stoi /
std::stof edge cases (trailing text, hex, inf, out-of-range), and the
frame-completeness rule.  Where the reference tree is mounted, the
reference's own example decks (input/*.params) are added as parsed tables.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from parrelray_b200 import build  # noqa: E402

DECKS = {
    "quirks": "\n".join([
        "a comment line without markers is skipped",
        "_tracer_",
        "<solver> = <rkf>\t\t\t#Euler or RG4",
        "<hmin> = <0.0001>",
        "<eps> = <1e-3>",
        "<bimage1> = <input/bin_back.ppm>   # a value with an underscore opens a block",
        "<after> = <x>",
        "_spacetime_",
        "<mass> = < 1.5 >",
        "<spin> = <0.9abc>",
        "<bad> = <abc>",
        "<big> = <99999999999>",
        "<huge> = <1e50>",
        "<tiny> = <1e-50>",
        "<neg> = <-3>",
        "<hex> = <0x10>",
        "<inf> = <inf>",
        "<empty> = <>",
        "noequals <k> <v>",
        "<k2> <v2> =",
        "= <orphan>",
        "<nokeyclose = <v3>",
        "<k4> = <v4",
        ">k5< = <v5>",
        "<dup> = <1>",
        "<dup> = <2>",
        "_",
        "<in_bare> = <1>",
        "__",
        "<in_empty> = <2>",
        "_a_b_c_",
        "<x> = <1>",
        "  _camera_  trailing",
        "<width> = <320>",
        "<w2> = <3.7>",
        "<SSAA> = <regular>",
        "_frame0_",
        "<x> = <30>", "<y> = <0>", "<z> = <0>", "<a> = <180>",
        "_frame1_",
        "<x> = <30>", "<y> = <0>", "<z> = <0>", "<a> = <180>", "<b> = <0>",
        "",
    ]),
    "crlf_frames": "\r\n".join([
        "_tracer_", "<solver> = <euler>", "<h> = <0.02>",
        "_camera_", "<width> = <64>", "<height> = <36>",
        "_frame0_", "<x> = <25>", "<y> = <0>", "<z> = <4.3>", "<a> = <180>", "<b> = <-10>",
        "_frame1_", "<x> = <24>", "<y> = <1>", "<z> = <4>", "<a> = <181>", "<b> = <-11>", "<mass> = <2>",
        "_frame2_", "<x> = <23>", "<y> = <2>", "<z> = <3.5>", "<a> = <182>", "<b> = <-12>",
        "_frame4_", "<x> = <1>", "<y> = <2>", "<z> = <3>", "<a> = <4>", "<b> = <5>",
        "_sphere0_", "<tex> = <tex1.ppm>", "<x0> = <10>", "<y0> = <0>", "<z0> = <0>", "<r0> = <1>",
        "<x1> = <9>", "<r2> = <1.5>",
        "_sphere1_", "<x0> = <-10>", "<y0> = <5>", "<z0> = <1>", "<r0> = <2>",
        "_sphere3_", "<x0> = <0>", "",
    ]),
}

QUERIES = [
    ("tracer", "solver"), ("tracer", "hmin"), ("tracer", "eps"), ("tracer", "h"), ("tracer", "bimage1"),
    ("back.ppm>   # a value with an underscore opens a block", "after"), ("spacetime", "mass"),
    ("spacetime", "spin"), ("spacetime", "bad"), ("spacetime", "big"), ("spacetime", "huge"),
    ("spacetime", "tiny"), ("spacetime", "neg"), ("spacetime", "hex"), ("spacetime", "inf"),
    ("spacetime", "empty"), ("spacetime", "dup"), ("spacetime", "missing"), ("nosuchblock", "x"),
    ("", "in_bare"), ("", "in_empty"), ("b", "x"), ("camera", "width"), ("camera", "w2"), ("camera", "SSAA"),
    ("frame0", "x"), ("frame1", "b"), ("frame1", "mass"), ("frame4", "a"), ("sphere0", "x1"), ("sphere0", "r2"),
    ("sphere0", "tex"), ("sphere1", "r0"), ("sphere3", "x0"),
]


def f32(x: float):
    if math.isnan(x):
        return "nan"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return x


class RefParser:
    def __init__(self):
        lib = C.CDLL(str(REPO / "oracle" / "_ref" / "libprr_ref_schw.so"))
        lib.prr_ref_parse.argtypes = [C.c_char_p]
        lib.prr_ref_has_block.argtypes = [C.c_char_p]
        lib.prr_ref_has.argtypes = [C.c_char_p, C.c_char_p]
        lib.prr_ref_par.restype = C.c_size_t
        lib.prr_ref_par.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]
        lib.prr_ref_pari.argtypes = [C.c_char_p, C.c_char_p]
        lib.prr_ref_parf.restype = C.c_float
        lib.prr_ref_parf.argtypes = [C.c_char_p, C.c_char_p]
        lib.prr_ref_parf_d.restype = C.c_float
        lib.prr_ref_parf_d.argtypes = [C.c_char_p, C.c_char_p, C.c_float]
        lib.prr_ref_entry.argtypes = [C.c_int, C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]
        self.lib = lib

    def table(self, text: str) -> dict:
        with tempfile.NamedTemporaryFile("wb", suffix=".params", delete=False) as f:
            f.write(text.encode())
            path = f.name
        lib = self.lib
        lib.prr_ref_parse(path.encode())
        Path(path).unlink()
        entries = []
        b, k, v = (C.create_string_buffer(4096) for _ in range(3))
        for i in range(lib.prr_ref_entry_count()):
            assert lib.prr_ref_entry(i, b, k, v, 4096) == 0
            entries.append([b.value.decode(), k.value.decode(), v.value.decode()])
        queries = []
        for blk, key in QUERIES:
            be, ke = blk.encode(), key.encode()
            n = lib.prr_ref_par(be, ke, None, 0)
            buf = C.create_string_buffer(n + 1)
            lib.prr_ref_par(be, ke, buf, n + 1)
            queries.append({"block": blk, "key": key, "has": lib.prr_ref_has(be, ke), "par": buf.value.decode(),
                            "pari": lib.prr_ref_pari(be, ke), "parf": f32(lib.prr_ref_parf(be, ke)),
                            "parf_default": f32(lib.prr_ref_parf_d(be, ke, C.c_float(7.5)))})
        blocks = sorted({e[0] for e in entries} | {q[0] for q in QUERIES})
        return {"entries": entries, "queries": queries,
                "has_block": {b_: lib.prr_ref_has_block(b_.encode()) for b_ in blocks},
                "check_frame": lib.prr_ref_check_frame()}


def main() -> int:
    build.build_reference()
    rp = RefParser()
    out = {"source": "reference readParams/par/pari/parf/headerExists/parExists/checkFrame (host build)",
           "decks": DECKS, "results": {name: rp.table(text) for name, text in DECKS.items()}}
    tree = build.reference_tree()
    ref_inputs = tree / "input" if tree else None
    if ref_inputs and ref_inputs.exists():
        # the reference's example decks, parsed by the reference (tables only)
        for p in sorted(ref_inputs.glob("*.params")):
            out["results"]["reference_" + p.stem] = rp.table(p.read_text(encoding="utf-8", errors="surrogateescape"))
    (HERE / "decks.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(f"wrote {HERE / 'decks.json'}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
