"""Host-side logic of the drop-in boundary (no GPU): parameters / -template, TIFF I/O,
the xprecon command line and its exit codes, and the product's geometry and planners
against the oracle."""
import ctypes as C
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.cases import CASES, make_case
from xpulse_recon_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "xpulse_recon_b200", "lib", "xprecon")


@pytest.fixture(scope="module")
def L():
    lib = _lib.lib()
    lib.xpr_template_json.restype = C.c_int64
    lib.xpr_template_json.argtypes = [C.c_char_p, C.c_uint64]
    lib.xpr_params_normalize.restype = C.c_int
    lib.xpr_params_normalize.argtypes = [C.c_char_p, C.c_char_p, C.c_uint64, C.POINTER(C.c_int64)]
    lib.xpr_tiff_write.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32]
    lib.xpr_tiff_read.argtypes = [C.c_char_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    lib.xpr_plan_chunks.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_float, C.c_void_p,
                                    C.c_int, C.POINTER(C.c_int)]
    lib.xpr_cull_layer.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int, C.c_void_p,
                                   C.c_void_p, C.POINTER(C.c_int)]
    return lib


def normalize(L, text):
    buf = C.create_string_buffer(1 << 16)
    n = C.c_int64()
    rc = L.xpr_params_normalize(text.encode(), buf, len(buf), C.byref(n))
    return rc, buf.value.decode()


def test_template_has_the_reference_schema(L):
    n = L.xpr_template_json(None, 0)
    buf = C.create_string_buffer(n + 1)
    L.xpr_template_json(buf, n + 1)
    t = json.loads(buf.value.decode())
    # global_parameters.hpp:8-54, specialized_parameters.hpp:22-39 (keys and defaults)
    r = t["recon"]
    assert r["input"] == "./" and r["output"] == "./recon/" and r["proj_output"] == ""
    assert r["method"] == "method_1b" and r["it"] == 1 and r["sit"] == 10 and r["mlog"] is True
    assert r["weight"] == 1.0 and abs(r["weight_factor"] - 0.9) < 1e-7 and r["normalize"] is False
    assert r["simulation"] is False
    g = t["geometry"]
    assert (g["so"], g["sd"], g["angle"], g["heli_offset"], g["heli_step"], g["angle_list"]) == (100, 1000, 360, 0, 1, [])
    d = t["detector"]
    assert abs(d["px"] - 0.1) < 1e-7 and (d["rx"], d["sx"], d["sy"], d["module_number"]) == (0, 0, 0, 1)
    assert d["module_angle_offset"] is None and d["module_center_offset_z"] == 0
    assert t["method2"]["overlap_fct"] == 1
    assert set(t["hartmann"]) == {"devx", "devy", "iterations", "iterations_fct", "iterations_step", "method"}
    assert set(t["ipr"]) == {"iterations", "iterations_fct", "iterations_step", "energy_kev"}


def test_parameters_accept_readme_style_json(L):
    # README.md:50-85 style: comments, trailing commas, images_preproc alias, modules[]
    text = """{
        "recon" : { "input" : "./in/", "method" : "naive", "it" : 2, "sit" : 5, // comment
                    "images_preproc" : true, },
        "geometry" : { "so" : 50.0, "sd" : 500.0, "angle" : 200.0, /* block */ },
        "detector" : { "px" : 0.2, "rx" : 1.5, "sx" : -2, "sy" : 3, "module_number" : 2,
                       "modules" : [ {"roll" : 1.0}, {"pitch": -0.5, "offset_x": 2} ] },
        "method2" : { "overlap_fct" : 7.0 },
    }"""
    rc, out = normalize(L, text)
    assert rc == 0, out
    p = json.loads(out)
    assert p["recon"]["method"] == "naive" and p["recon"]["it"] == 2 and p["recon"]["sit"] == 5
    assert p["recon"]["normalize"] is True
    assert p["geometry"]["angle"] == 200.0 and p["detector"]["module_number"] == 2
    assert p["detector"]["rx"] == 1.5  # kept in pixels; converted with px where the geometry is built
    assert p["detector"]["modules"][0]["roll"] == 1.0 and p["detector"]["modules"][1]["offset_x"] == 2.0
    assert p["method2"]["overlap_fct"] == 1.0  # parameters.hpp:35 clamps to [0.01, 1]


def test_resume_keys_round_trip(L):
    rc, out = normalize(L, '{"recon": {"it": 4, "resume": "./recon/", "first_iteration": 3}}')
    assert rc == 0, out
    r = json.loads(out)["recon"]
    assert r["resume"] == "./recon/" and r["first_iteration"] == 3
    rc, out = normalize(L, '{"recon": {"it": 4}}')
    assert "resume" not in json.loads(out)["recon"]


@pytest.mark.parametrize("text", ['{"recon": {"method": "bogus"}}', '{"recon": {"it": "x"}}', '{"recon": ', "[1, 2]",
                                  '{"detector": {"module_number": 2, "modules": [{}]}}',
                                  '{"recon": {"it": 2, "first_iteration": 2}}',
                                  '{"recon": {"it": 2, "first_iteration": -1}}',
                                  '{"recon": {"it": 3, "first_iteration": 1.5}}'])
def test_bad_parameters_are_rejected(L, text):
    rc, msg = normalize(L, text)
    assert rc == 6, msg  # XPR_ERR_PARAM


def test_tiff_roundtrip_and_big_endian(L, tmp_path):
    rng = np.random.default_rng(0)
    img = rng.normal(size=(13, 29)).astype(np.float32)
    p = str(tmp_path / "a.tif")
    assert L.xpr_tiff_write(p.encode(), img.ctypes.data, 29, 13) == 0
    out = np.zeros_like(img)
    w, h = C.c_uint32(), C.c_uint32()
    assert L.xpr_tiff_read(p.encode(), out.ctypes.data, out.size, C.byref(w), C.byref(h)) == 0
    assert (w.value, h.value) == (29, 13)
    np.testing.assert_array_equal(out.view(np.uint32), img.view(np.uint32))
    # a big-endian, two-strip float TIFF written by hand from the TIFF 6.0 layout
    H, W = 5, 3
    data = np.arange(H * W, dtype=np.float32) * 0.5 - 2.0
    be = data.astype(">f4").tobytes()
    entries = [(256, 3, 1, W), (257, 3, 1, H), (258, 3, 1, 32), (259, 3, 1, 1), (262, 3, 1, 1),
               (273, 4, 2, 0), (277, 3, 1, 1), (278, 3, 1, 3), (279, 4, 2, 0), (339, 3, 1, 3)]
    ifd_off = 8
    arrays_off = ifd_off + 2 + 12 * len(entries) + 4
    strip0 = arrays_off + 16
    strip1 = strip0 + 3 * W * 4
    hdr = bytearray(b"MM" + struct.pack(">HI", 42, ifd_off))
    hdr += struct.pack(">H", len(entries))
    for tag, typ, cnt, val in entries:
        if tag == 273:
            hdr += struct.pack(">HHII", tag, typ, cnt, arrays_off)
        elif tag == 279:
            hdr += struct.pack(">HHII", tag, typ, cnt, arrays_off + 8)
        elif typ == 3:
            hdr += struct.pack(">HHIHH", tag, typ, cnt, val, 0)
        else:
            hdr += struct.pack(">HHII", tag, typ, cnt, val)
    hdr += struct.pack(">I", 0)
    hdr += struct.pack(">II", strip0, strip1) + struct.pack(">II", 3 * W * 4, 2 * W * 4)
    q = tmp_path / "b.tif"
    q.write_bytes(bytes(hdr) + be)
    out = np.zeros(H * W, np.float32)
    assert L.xpr_tiff_read(str(q).encode(), out.ctypes.data, out.size, C.byref(w), C.byref(h)) == 0
    np.testing.assert_array_equal(out, data)
    # not a float TIFF / missing file
    assert L.xpr_tiff_read(str(tmp_path / "none.tif").encode(), None, 0, None, None) == 5


def test_cli_exit_codes_without_gpu(tmp_path):
    assert os.path.exists(CLI)
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode == 255 and "template" in r.stdout  # -1
    r = subprocess.run([CLI, "-template"], capture_output=True, text=True)
    assert r.returncode == 0 and json.loads(r.stdout)["recon"]["method"] == "method_1b"
    r = subprocess.run([CLI, '{"recon": {"method": "nope"}}'], capture_output=True, text=True)
    assert r.returncode == 254  # -2
    r = subprocess.run([CLI, str(tmp_path / "missing.json")], capture_output=True, text=True)
    assert r.returncode == 254
    empty = tmp_path / "empty"
    empty.mkdir()
    cfg = {"recon": {"input": str(empty), "output": str(tmp_path / "out"), "method": "naive"}}
    r = subprocess.run([CLI, json.dumps(cfg)], capture_output=True, text=True)
    assert r.returncode == 253 and "No valid TIFF" in r.stderr  # -3


def _product_geometry(gp, fp64):
    """xpr_geometry with the oracle's parameter struct (same layout)."""
    L = _lib.lib()
    out = np.zeros((gp.projections * gp.module_number, 20), np.float32)
    go = _lib.GeomOut()
    g = _lib.GeomParams()
    C.memmove(C.byref(g), C.byref(gp), C.sizeof(g))
    assert L.xpr_geometry(C.byref(g), int(fp64), out.ctypes.data, C.byref(go)) == 0
    return out, go


@pytest.mark.parametrize("fp64", [False, True])
@pytest.mark.parametrize("name", sorted(CASES))
def test_product_geometry_matches_oracle(name, fp64):
    c = make_case(name, fp64=fp64)
    out, go = _product_geometry(c["gp"], fp64)
    np.testing.assert_array_equal(out.view(np.uint32), c["pd_all"].view(np.uint32))
    assert (go.vx, go.vwidth, go.vheight, go.concurrent) == (c["go"].vx, c["go"].vwidth, c["go"].vheight,
                                                              c["go"].concurrent)
    assert list(go.orig) == list(c["go"].orig)


def test_fp64_geometry_is_close_to_fp32():
    c32 = make_case("offsets64", fp64=False)
    c64 = make_case("offsets64", fp64=True)
    rel = np.abs(c64["pd_all"] - c32["pd_all"]) / (np.abs(c32["pd_all"]) + 1e-3)
    assert rel.max() < 1e-4


@pytest.mark.parametrize("name,budget", [("offsets64", 1 << 30), ("offsets64", 900_000), ("plain48", 400_000),
                                         ("helical", 300_000), ("modules2", 350_000)])
def test_chunk_planner_matches_oracle(L, name, budget):
    c = make_case(name)
    gp, go = c["gp"], c["go"]
    a = np.zeros((256, 6), np.int64)
    b = np.zeros((256, 6), np.int64)
    n_o = O.lib().orc_plan_chunks(C.byref(gp), C.byref(go), c["pd_all"], budget, budget, 1.0, b, 256)
    n_p = C.c_int()
    g = _lib.GeomParams()
    C.memmove(C.byref(g), C.byref(gp), C.sizeof(g))
    go2 = _lib.GeomOut()
    C.memmove(C.byref(go2), C.byref(go), C.sizeof(go2))
    assert L.xpr_plan_chunks(C.byref(g), C.byref(go2), c["pd_all"].ctypes.data, budget, budget, 1.0, a.ctypes.data,
                             256, C.byref(n_p)) == 0
    assert n_p.value == n_o
    if n_o > 0:
        np.testing.assert_array_equal(a[:n_o], b[:n_o])
        assert (a[:n_o, 1] >= 0).all() and a[0, 0] >= 0


@pytest.mark.parametrize("name", ["offsets64", "plain48", "modules2", "helical"])
def test_culling_matches_oracle(L, name):
    c = make_case(name)
    gp, go = c["gp"], c["go"]
    g = _lib.GeomParams()
    C.memmove(C.byref(g), C.byref(gp), C.sizeof(g))
    go2 = _lib.GeomOut()
    C.memmove(C.byref(go2), C.byref(go), C.sizeof(go2))
    for sit in range(gp.sit):
        for layer in range(0, int(go.vheight), 7):
            a1, a2 = np.zeros(512, np.uint16), np.zeros(512, np.uint16)
            b1, b2 = np.zeros(512, np.uint16), np.zeros(512, np.uint16)
            n = C.c_int()
            pm = int(gp.module_number > 1)
            assert L.xpr_cull_layer(C.byref(g), C.byref(go2), c["pd_all"].ctypes.data, sit, layer, pm, a1.ctypes.data,
                                    a2.ctypes.data, C.byref(n)) == 0
            m = O.lib().orc_cull_layer(C.byref(gp), C.byref(go), c["pd_all"], sit, layer, pm, b1, b2)
            assert n.value == m
            np.testing.assert_array_equal(a1[:m], b1[:m])
            np.testing.assert_array_equal(a2[:m], b2[:m])


def test_strict_walk_division_and_pixel_rule_on_the_cpu(tmp_path):
    """The STRICT column walk divides by a column's n_w with a reciprocal, its residual and
    one Markstein correction, and rounds half away from zero with two round-toward-zero
    adds (xpr_kernels.cu: div_exact, pix_bits2).  The same operations in C on the host
    (hardware fma, IEEE division) must give the IEEE quotient and the reference's pixel
    on 10^8 operand pairs (half of them at rounding midpoints) and 2 x 10^7 pixel
    decisions around half-integer borders; the GPU parity tests then show the kernels
    equal to the reference bit for bit."""
    src = os.path.join(os.path.dirname(os.path.abspath(__file__)), "exact_div_check.c")
    exe = str(tmp_path / "exact_div_check")
    r = subprocess.run(["gcc", "-O2", "-mfma", "-fopenmp", "-ffp-contract=off", "-frounding-math", "-o", exe, src,
                        "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe, "2000", "50000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    res = {line.split()[0]: (int(line.split()[1]), int(line.split()[2])) for line in out.stdout.splitlines()}
    assert res["division"][0] == 2000 * 50000 and res["division"][1] == 0, res
    assert res["pixel"][0] == 20000000 and res["pixel"][1] == 0, res
