"""Generate the committed golden fixtures under tests/golden/ (run here, where
the reference tree exists; the fixtures travel, the reference does not).

    python tests/golden/make_golden.py

refcpu_frames.json  FNV-1a 64 hashes of every frame the reference's own
                    compiled CPU reconstruction (oracle/_ref: vp9_reconstruct.c
                    + vp9_frame.c, driven with the pool rules of
                    vp9_decoder.c:224-231) produces for seeded synthetic
                    streams.
spec_frames.json    the same for the SPEC restatement (oracle/), so its output
                    is frozen against accidental change.
layout.json         sizeof/offsetof of the boundary structs as the reference
                    headers compile them.
tables.json         SHA-256 of the quantiser tables, the regular 8-tap filter and
                    the intra-mode -> transform-type map as the reference
                    sources spell them (src/decoder/vp9_dequant.h:12-60,
                    shaders/vp9_mc.comp.glsl:40-57,
                    src/decoder/vp9_default_probs.h:1728).
spec_idct.json      input/output vectors of the shader inverse transforms,
                    computed by a mechanical translation of
                    shaders/vp9_idct.comp.glsl's idct4/8/16/32 functions and
                    its main() dequant/shift logic into Python (done here at
                    generation time; only the vectors are committed).
spec_intra.json     the shader intra predictor (shaders/vp9_intra_pred.comp.glsl
                    main() and its sample_* helpers, translated statement by
                    statement by glsl_py.py and run per invocation of a 32x32
                    workgroup): every block size, the four modes it implements
                    and two it does not, at the four edge-availability cases;
                    inputs from tests/golden/vectors.py seeds, outputs as
                    digests of the predicted plane.
spec_mc.json        the shader luma motion compensation (shaders/vp9_mc.comp.glsl
                    main() and fetch_ref, translated the same way, run per
                    pixel of a 64x48 frame with one MV in every 4x4 cell): all
                    64 (x, y) phase pairs and MVs far outside the frame.
"""
import ctypes as C
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# the reference tree: $CVP9_REFERENCE, else a checkout named "reference"
# beside this repository
REF = os.environ.get("CVP9_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from compute_vp9_b200 import Synth, fnv1a64, synth_config  # noqa: E402
from compute_vp9_b200.cvp9_ctypes import layout_offsets  # noqa: E402
from oracle import oracle_py as O  # noqa: E402

# (name, preset, w, h, frames, seed, overrides)
CASES = [
    ("c1_small", 1, 320, 192, 4, 11, {}),
    ("c2_small", 2, 352, 288, 6, 11, {"gop": 3}),
    ("edges_sub8", 2, 200, 120, 5, 11, {"gop": 2, "min_bsize": 4, "skip_prob": 0.2,
                                        "all_intra_modes": 1, "intra_in_inter": 0.3}),
    ("odd_tiles", 2, 250, 130, 4, 11, {"gop": 2, "log2_tile_cols": 1, "sharpness": 5}),
    ("big_tx", 2, 256, 256, 4, 11, {"gop": 2, "tx_weights": [0, 0, 20, 80], "density_max": 0.5}),
    ("lf_zero", 1, 192, 128, 3, 11, {"lf_level": 0}),
    ("c1_720p", 1, 1280, 720, 2, 11, {}),
]


def frame_hashes(stream, syn, n):
    return ["%016x" % fnv1a64(stream.decode(syn.frame(f))) for f in range(n)]


def table_hash():
    t = open(os.path.join(REF, "src/decoder/vp9_dequant.h")).read()
    vals = []
    for name in ("vp9_dc_qlookup", "vp9_ac_qlookup"):
        m = re.search(name + r"\[256\] = \{(.*?)\};", t, re.S)
        vals.append([int(x) for x in m.group(1).replace("\n", " ").split(",") if x.strip()])
    g = open(os.path.join(REF, "shaders/vp9_mc.comp.glsl")).read()
    m = re.search(r"SUBPEL_FILTER\[16\]\[8\] = int\[16\]\[8\]\((.*?)\);", g, re.S)
    rows = re.findall(r"int\[8\]\(([^)]*)\)", m.group(1))
    filt = [[int(x) for x in r.split(",")] for r in rows]
    d = open(os.path.join(REF, "src/decoder/vp9_default_probs.h")).read()
    m = re.search(r"vp9_intra_mode_to_tx_type\[10\] = \{([^}]*)\}", d)
    txt = [int(x) for x in m.group(1).split(",")]
    return {
        "intra_tx_type_sha256": hashlib.sha256(np.array(txt, np.int32).tobytes()).hexdigest(),
        "dc_q_sha256": hashlib.sha256(np.array(vals[0], np.int32).tobytes()).hexdigest(),
        "ac_q_sha256": hashlib.sha256(np.array(vals[1], np.int32).tobytes()).hexdigest(),
        "subpel_regular_sha256": hashlib.sha256(np.array(filt, np.int32).tobytes()).hexdigest(),
    }


def glsl_idct_functions():
    """Translate idct4_c..idct32_c from the shader source into Python source."""
    g = open(os.path.join(REF, "shaders/vp9_idct.comp.glsl")).read()
    out = []
    for n in (4, 8, 16, 32):
        m = re.search(r"void idct%d_c\(int input_arr\[%d\], inout int output_arr\[%d\]\) \{(.*?)\n\}" % (n, n, n), g, re.S)
        body = m.group(1)
        body = body.replace("shared_step1[gl_LocalInvocationID.x]", "s1").replace(
            "shared_step2[gl_LocalInvocationID.x]", "s2")
        lines = ["def idct%d(input_arr):" % n, "    s1 = [0]*32; s2 = [0]*32; output_arr = [0]*%d" % n]
        for ln in body.split("\n"):
            ln = ln.strip()
            if not ln or ln.startswith("//") or ln.startswith("int temp1"):
                continue
            ln = ln.rstrip(";")
            ln = re.sub(r"input_arr\[(\d+) / 2\]", r"input_arr[\1 // 2]", ln)
            ln = re.sub(r"ROUND_SHIFT\((.*)\)$", r"RS(\1)", ln)
            lines.append("    " + ln)
        lines.append("    return output_arr")
        out.append("\n".join(lines))
    return "\n\n".join(out)


def wrap32(v):
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v & 0x80000000 else v


def spec_vectors():
    src = glsl_idct_functions()
    ns = {}

    def RS(x):
        return wrap32(wrap32(x) + 8192) >> 14
    ns["RS"] = RS
    # the shader arithmetic is 32-bit: wrap every assignment
    src = re.sub(r"(s[12]\[\d+\]|output_arr\[\d+\]|temp[12]) = (.*)", r"\1 = W(\2)", src)
    ns["W"] = wrap32
    exec(src, ns)
    rng = np.random.default_rng(2024)
    vecs = []
    for n in (4, 8, 16, 32):
        fn = ns["idct%d" % n]
        for trial in range(6):
            dens = [0.05, 0.3, 1.0][trial % 3]
            x = np.where(rng.random((n, n)) < dens, rng.integers(-512, 513, (n, n)), 0).astype(np.int64)
            if trial == 5:
                x[:] = rng.integers(-32768, 32768, (n, n))   # extreme: exercises 32-bit wrap
            qdc, qac = [(57, 67), (4, 4), (1336, 1828)][trial % 3]
            buf = [[0] * n for _ in range(n)]
            for c in range(n):
                col = [wrap32(int(x[r, c]) * (qdc if (r == 0 and c == 0) else qac)) for r in range(n)]
                o = fn(col)
                for r in range(n):
                    buf[r][c] = o[r]
            for r in range(n):
                buf[r] = fn(buf[r])
            sh = {4: 4, 8: 5, 16: 6, 32: 6}[n]
            res = [[wrap32(buf[r][c] + (1 << (sh - 1))) >> sh for c in range(n)] for r in range(n)]
            vecs.append({"n": n, "q_dc": qdc, "q_ac": qac, "in": x.astype(int).tolist(), "out": res})
    return vecs


class _Obj:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def _shader_namespace(shader, functions):
    """Execute the translated shader functions in a namespace with the GLSL
    built-ins they use."""
    import glsl_py
    src = open(os.path.join(REF, "shaders", shader)).read()
    code = "".join(glsl_py.translate(src, f) for f in functions)

    def clamp(v, lo, hi):
        if isinstance(v, tuple):
            return tuple(min(max(a, b), c) for a, b, c in zip(v, lo, hi))
        return min(max(v, lo), hi)

    def vec2(*a):
        return (a[0], a[0]) if len(a) == 1 else tuple(a)

    ns = {"u32": lambda v: int(v) & 0xFFFFFFFF, "i32": lambda v: wrap32(int(v)), "u8": lambda v: int(v) & 0xFF,
          "clamp": clamp, "vec2": vec2}
    exec(code, ns)
    return ns


def spec_intra_vectors():
    from vectors import INTRA_PLANE, digest, intra_cases, plane_bytes
    ns = _shader_namespace("vp9_intra_pred.comp.glsl", ("sample_above", "sample_left", "sample_top_left", "main"))
    out = []
    for case in intra_cases():
        plane = plane_bytes(case["seed"], INTRA_PLANE)
        stride = INTRA_PLANE[1]
        ns["pred"] = plane.reshape(-1).astype(int).tolist()
        ns["blocks"] = [_Obj(is_intra=1, skip=0, block_size=case["n"], tx_size=0, pred_mode=case["mode"],
                             qstep=0, coeff_offset=0, dst_stride=stride,
                             dst_offset=case["y"] * stride + case["x"], qstep_dc=0)]
        ns["gl_WorkGroupID"] = (0, 0, 0)
        for py in range(32):
            for px in range(32):
                ns["gl_LocalInvocationID"] = (px, py)
                ns["main"]()
        got = np.array(ns["pred"], np.uint8).reshape(INTRA_PLANE)
        out.append(dict(case, digest=digest(got)))
    return out


def spec_mc_vectors():
    from vectors import MC_PLANE, digest, mc_cases, plane_bytes
    ns = _shader_namespace("vp9_mc.comp.glsl", ("fetch_ref", "main"))
    g = open(os.path.join(REF, "shaders/vp9_mc.comp.glsl")).read()
    m = re.search(r"SUBPEL_FILTER\[16\]\[8\] = int\[16\]\[8\]\((.*?)\);", g, re.S)
    ns["SUBPEL_FILTER"] = [[int(x) for x in r.split(",")] for r in re.findall(r"int\[8\]\(([^)]*)\)", m.group(1))]
    h, w = MC_PLANE
    ns["pc"] = _Obj(frame_width=w, frame_height=h, block_size=0, filter_type=0)
    out = []
    for case in mc_cases():
        ref = plane_bytes(case["seed"], MC_PLANE)
        tex = _Obj(data=ref)

        def texel_fetch(t, p, lod):
            return _Obj(r=float(t.data[p[1], p[0]]) / 255.0)
        ns["texelFetch"] = texel_fetch
        ns["ref_frames"] = [tex, tex, tex]
        cells = ((w + 3) // 4) * ((h + 3) // 4)
        ns["mv"] = [(case["mvx"], case["mvy"], 0, 0)] * cells
        ns["dst_luma"] = [0] * (w * h)
        for py in range(h):
            for px in range(w):
                ns["gl_GlobalInvocationID"] = (px, py)
                ns["main"]()
        out.append(dict(case, digest=digest(np.array(ns["dst_luma"], np.uint8))))
    return out


def main():
    O.build()
    if not O.ref_available():
        raise SystemExit("oracle/_ref not built: needs the reference sources at %s" % REF)
    ref, spec = {}, {}
    for name, preset, w, h, n, seed, ov in CASES:
        cfg = dict(preset=preset, w=w, h=h, frames=n, seed=seed, overrides=ov)
        ref[name] = dict(cfg, hashes=frame_hashes(O.RefStream(), Synth(synth_config(preset, w, h, seed, **ov)), n))
        spec[name] = dict(cfg, hashes=frame_hashes(O.OracleStream(O.SPEC),
                                                   Synth(synth_config(preset, w, h, seed, **ov)), n))
    json.dump(ref, open(os.path.join(HERE, "refcpu_frames.json"), "w"), indent=1)
    json.dump(spec, open(os.path.join(HERE, "spec_frames.json"), "w"), indent=1)
    buf = (C.c_uint32 * 64)()
    k = O.ref_lib().ref_layout(buf, 64)
    json.dump({"offsets": list(buf[:k])}, open(os.path.join(HERE, "layout.json"), "w"))
    json.dump(table_hash(), open(os.path.join(HERE, "tables.json"), "w"), indent=1)
    json.dump(spec_vectors(), open(os.path.join(HERE, "spec_idct.json"), "w"))
    json.dump(spec_intra_vectors(), open(os.path.join(HERE, "spec_intra.json"), "w"), indent=0)
    json.dump(spec_mc_vectors(), open(os.path.join(HERE, "spec_mc.json"), "w"), indent=0)
    print("golden fixtures written; layout match:", list(buf[:k]) == layout_offsets())


if __name__ == "__main__":
    main()
