"""The C ABI library: it builds for sm_100a, exports every entry point that
include/morphompm_b200.h declares, its struct layouts agree with the ctypes
mirror, and host-only plan construction validates its arguments.  No CUDA
calls are made here."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from morphompm_b200 import _lib as L
from morphompm_b200.build import ROOT

HEADER = os.path.join(ROOT, "include", "morphompm_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|int64_t)\s+\**(mpm_\w+)\s*\(", src, re.M)))


def test_exports_every_declared_symbol():
    lib = L.load()
    names = declared()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(L.EXPORTS), set(names) ^ set(L.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", L.lib_path()], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


def test_struct_layout_matches_ctypes():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "morphompm_b200.h"
#define O(T, f) printf(#T "." #f " %zu\n", offsetof(T, f))
int main(void) {
  printf("MpmScene %zu\nMpmParticles %zu\nMpmCotangents %zu\nMpmTuning %zu\n", sizeof(MpmScene),
         sizeof(MpmParticles), sizeof(MpmCotangents), sizeof(MpmTuning));
  O(MpmScene, p_begin); O(MpmScene, wall); O(MpmScene, growth_mode); O(MpmScene, dx); O(MpmScene, gravity);
  O(MpmScene, mu); O(MpmScene, kappa); O(MpmScene, eps); O(MpmScene, growth_A); O(MpmScene, ramp_steps);
  O(MpmParticles, Fg); O(MpmParticles, sc9); O(MpmCotangents, Fg); O(MpmTuning, fp64_gap_thresh); O(MpmTuning, tile_z);
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "layout")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(l.rsplit(" ", 1) for l in out if l)
    assert int(got["MpmScene"]) == C.sizeof(L.MpmScene)
    assert int(got["MpmParticles"]) == C.sizeof(L.MpmParticles)
    assert int(got["MpmCotangents"]) == C.sizeof(L.MpmCotangents)
    assert int(got["MpmTuning"]) == C.sizeof(L.MpmTuning)
    for k, v in got.items():
        if "." in k:
            T, f = k.split(".")
            assert getattr(getattr(L, T), f).offset == int(v), k


def _scene(n, p0=0, shape=(8, 8, 8)):
    s = L.MpmScene()
    for d in range(3):
        s.shape[d] = shape[d]
    s.p_begin, s.p_end = p0, p0 + n
    s.dx, s.dt, s.damping, s.pmass, s.vol0 = 0.1, 1e-3, 0.05, 8e-3, 8e-6
    return s


def test_plan_host_validation():
    lib = L.load()
    arr = (L.MpmScene * 2)(_scene(100), _scene(50, 100, (5, 6, 7)))
    h = C.c_void_p()
    assert lib.mpm_plan_create(arr, 2, 8, None, C.byref(h)) == L.MPM_OK
    nb = C.c_size_t()
    assert lib.mpm_plan_workspace_bytes(h, C.byref(nb)) == 0 and nb.value > 0
    tb = C.c_size_t()
    assert lib.mpm_plan_tape_bytes(h, C.byref(tb)) == 0 and 0 < tb.value < nb.value
    assert lib.mpm_plan_num_particles(h) == 150
    lib.mpm_plan_destroy(h)
    # particle ranges must tile [0, n) in scene order
    bad = (L.MpmScene * 2)(_scene(100), _scene(50, 90))
    assert lib.mpm_plan_create(bad, 2, 8, None, C.byref(h)) == L.MPM_ERR_ARG
    assert lib.mpm_plan_create(arr, 2, 2, None, C.byref(h)) == L.MPM_ERR_ARG
    s = _scene(10)
    s.model = 7
    assert lib.mpm_plan_create((L.MpmScene * 1)(s), 1, 8, None, C.byref(h)) == L.MPM_ERR_ARG
    # null pointers are rejected before any CUDA call
    assert lib.mpm_step_fwd(None, None, None, 1, 0, None, None) == L.MPM_ERR_ARG
    assert lib.mpm_stress(None, 8, 1, None, None, None, None, None) == L.MPM_ERR_ARG


def test_tape_grows_with_tile_cap():
    lib = L.load()
    arr = (L.MpmScene * 1)(_scene(1000, 0, (64, 64, 64)))
    sizes = []
    for cap in (0, 10):
        t = L.MpmTuning()
        t.active_tile_cap = cap
        h = C.c_void_p()
        assert lib.mpm_plan_create(arr, 1, 4, C.byref(t), C.byref(h)) == 0
        tb = C.c_size_t()
        lib.mpm_plan_tape_bytes(h, C.byref(tb))
        sizes.append(tb.value)
        lib.mpm_plan_destroy(h)
    assert sizes[1] < sizes[0]


def test_rollout_workspace_layout():
    """mpm_rollout_workspace_bytes (host only): k+1 segment states, 2 cotangent
    slabs and k tapes; with recompute also ceil(N/k) checkpoints and 2 scratch
    states.  Calls that would launch are refused on bad arguments first."""
    lib = L.load()
    arr = (L.MpmScene * 1)(_scene(1000, 0, (16, 16, 16)))
    h = C.c_void_p()
    assert lib.mpm_plan_create(arr, 1, 4, None, C.byref(h)) == 0
    tb = C.c_size_t()
    lib.mpm_plan_tape_bytes(h, C.byref(tb))
    up = lambda b: (b + 255) // 256 * 256
    slab, tape = up(24 * 1000 * 4), up(tb.value)

    def ws(n, k):
        nb = C.c_size_t(7)
        assert lib.mpm_rollout_workspace_bytes(h, n, k, C.byref(nb)) == 0
        return nb.value

    assert ws(0, 0) == 0
    assert ws(10, 0) == ws(10, 10) == ws(10, 99) == (11 + 2) * slab + 10 * tape
    assert ws(10, 4) == (3 + 5 + 2 + 2) * slab + 4 * tape
    assert ws(10, 1) == (10 + 2 + 2 + 2) * slab + 1 * tape
    nb = C.c_size_t()
    assert lib.mpm_rollout_workspace_bytes(h, -1, 0, C.byref(nb)) == L.MPM_ERR_ARG
    assert lib.mpm_rollout_workspace_bytes(h, 5, -2, C.byref(nb)) == L.MPM_ERR_ARG
    # unbound plan (no workspace): refused before any CUDA call
    assert lib.mpm_rollout_fwd(h, 16, None, 3, 0, 1, None, 4096, None) == L.MPM_ERR_ARG
    assert lib.mpm_rollout_bwd(h, None, 16, 3, 0, 1, None, 4096, None, None, None, None) == L.MPM_ERR_ARG
    lib.mpm_plan_destroy(h)


def test_checked_build_exports_the_same_abi():
    """The bounds-checked library (MPM_CHECK_BOUNDS) exports exactly the
    release library's entry points; the release library reports that it has
    no checks."""
    from morphompm_b200 import build as B
    lib = L.load()
    cnt, site, idx = C.c_int64(5), C.c_int32(5), C.c_int64(5)
    assert lib.mpm_check_violations(C.byref(cnt), C.byref(site), C.byref(idx), None) == L.MPM_ERR_UNSUPPORTED
    assert (cnt.value, site.value, idx.value) == (0, 0, -1)
    path = B.build(checked=True)
    syms = lambda p: set(re.findall(r"\bT (mpm_\w+)", subprocess.run(["nm", "-D", "--defined-only", p],
                                                                     capture_output=True, text=True).stdout))
    assert syms(path) == syms(L.lib_path()) == set(declared())


def test_budget_schedule_covers_the_engine_memory():
    """The checkpoint interval budget_schedule picks fits: the native engine's
    workspace (mpm_rollout_workspace_bytes) plus the three slabs Rollout owns
    (final state, loss seed, initial cotangents) stay within the budget."""
    from morphompm_b200.trajectory import budget_schedule
    lib = L.load()
    n = 5000
    arr = (L.MpmScene * 1)(_scene(n, 0, (24, 24, 24)))
    h = C.c_void_p()
    assert lib.mpm_plan_create(arr, 1, 4, None, C.byref(h)) == 0
    tb = C.c_size_t()
    lib.mpm_plan_tape_bytes(h, C.byref(tb))
    state = 24 * n * 4
    for steps in (1, 7, 50, 200):
        for frac in (0.05, 0.3, 1.0, 3.0):
            budget = int(frac * steps * (state + tb.value))
            k = budget_schedule(steps, state, tb.value, budget)
            nb = C.c_size_t()
            assert lib.mpm_rollout_workspace_bytes(h, steps, k, C.byref(nb)) == 0
            used = nb.value + 3 * state
            if k > 1:                     # k = 1 is the floor, taken even when nothing fits
                assert used <= budget + 8 * 256, (steps, frac, k, used, budget)
    lib.mpm_plan_destroy(h)


def test_plan_refuses_grids_beyond_the_key_range():
    """Cell keys are 32-bit: a scene or batch with 2^31 or more padded cells is
    refused at plan creation (host only), not wrapped."""
    lib = L.load()
    h = C.c_void_p()
    big = _scene(10, 0, (2048, 2048, 2048))          # 2050^3 padded cells
    assert lib.mpm_plan_create((L.MpmScene * 1)(big), 1, 4, None, C.byref(h)) == L.MPM_ERR_ARG
    ok = _scene(10, 0, (1000, 1000, 1000))           # 1002^3 < 2^31
    assert lib.mpm_plan_create((L.MpmScene * 1)(ok), 1, 4, None, C.byref(h)) == L.MPM_OK
    lib.mpm_plan_destroy(h)
    three = (L.MpmScene * 3)(*(_scene(10, 10 * i, (1000, 1000, 1000)) for i in range(3)))
    assert lib.mpm_plan_create(three, 3, 4, None, C.byref(h)) == L.MPM_ERR_ARG    # 3 x 1.006e9


def test_noalloc_refuses_large_scenes_before_any_cuda_call():
    """mpm_step_fwd_noalloc sizes its layout on the host first: a scene that
    does not fit the fixed scratch, including one beyond the 32-bit cell keys,
    returns MPM_ERR_TOO_LARGE without touching the device (the particle
    pointers are never dereferenced on the host)."""
    lib = L.load()
    fake = L.MpmParticles()
    fake.x, fake.v, fake.C, fake.F, fake.Fg = 4096, 8192, 12288, 16384, 20480
    fake.sp3, fake.sc3, fake.sp9, fake.sc9 = 3, 1, 9, 1
    out = L.MpmParticles()
    out.x, out.v, out.C, out.F, out.Fg = 24576, 28672, 32768, 36864, 40960
    out.sp3, out.sc3, out.sp9, out.sc9 = 3, 1, 9, 1
    for shape in ((2048, 2048, 2048), (256, 256, 256)):
        sc = _scene(10, 0, shape)
        assert lib.mpm_step_fwd_noalloc(C.byref(sc), 4, C.byref(fake), C.byref(out), 1, 0, None, None) == \
            L.MPM_ERR_TOO_LARGE


def test_bin_keys_refuses_grids_beyond_int32_keys():
    lib = L.load()
    sc = _scene(10, 0, (2048, 2048, 2048))
    keys = (C.c_int32 * 10)()
    assert lib.mpm_bin_keys(C.byref(sc), 8, 10, C.c_void_p(4096), keys, None) == L.MPM_ERR_ARG
