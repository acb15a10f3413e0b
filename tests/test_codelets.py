"""Generated CUDA codelets, compiled for the host with g++, against the
reference's codelet evaluator (golden vectors) -- the role of the reference's
compiler/mofft_compiler/validate.py candidate harness."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from mofft_b200.codegen import gen_codelets
from tests.conftest import DBL_EPS, FLT_EPS, ROOT

RADICES = gen_codelets.RADICES


HARNESS = r"""
#define __device__
#define __forceinline__ inline
#include <cstdio>
#include <cstdlib>
#include "codelets.cuh"
template <typename T, int R> void run(const double* in, double* out) {
  T re[R], im[R];
  for (int i = 0; i < R; ++i) { re[i] = (T)in[2*i]; im[i] = (T)in[2*i+1]; }
  Dft<R>::fwd(re, im);
  for (int i = 0; i < R; ++i) { out[2*i] = (double)re[i]; out[2*i+1] = (double)im[i]; }
}
template <typename T, int R, int F> void runf(const double* in, double* out) {
  T re[R], im[R];
  for (int i = 0; i < R; ++i) { re[i] = (T)in[2*i]; im[i] = (T)in[2*i+1]; }
  DftFamily<R, F>::fwd(re, im);
  for (int i = 0; i < R; ++i) { out[2*i] = (double)re[i]; out[2*i+1] = (double)im[i]; }
}
template <typename T> void dispatch(int R, int F, const double* in, double* out) {
  if (F == 0) {
    switch (R) {
#define C(RR) case RR: run<T, RR>(in, out); break;
      C(2) C(3) C(4) C(5) C(6) C(7) C(8) C(9) C(10) C(11) C(12) C(13) C(14) C(15) C(16) C(32) C(64)
    }
    return;
  }
FAMILY_DISPATCH
}
int main(int argc, char** argv) {
  int bits, R, F;
  double in[128], out[128];
  while (scanf("%d %d %d", &bits, &R, &F) == 3) {
    for (int i = 0; i < 2 * R; ++i) if (scanf("%lf", &in[i]) != 1) return 1;
    if (bits == 32) dispatch<float>(R, F, in, out); else dispatch<double>(R, F, in, out);
    for (int i = 0; i < 2 * R; ++i) printf("%.17g ", out[i]);
    printf("\n");
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("codelets")
    cuh, _ = gen_codelets.generate()
    (d / "codelets.cuh").write_text(cuh)
    fam = []
    for radix in RADICES:
        for name in gen_codelets.FAMILIES:
            if gen_codelets.family_defined(radix, name):
                f = gen_codelets.FAMILY_ID[name]
                fam.append(f"  if (R == {radix} && F == {f}) {{ runf<T, {radix}, {f}>(in, out); "
                           "return; }")
    (d / "h.cpp").write_text(HARNESS.replace("FAMILY_DISPATCH", "\n".join(fam)))
    exe = d / "h"
    subprocess.run(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-o", str(exe),
                    str(d / "h.cpp")], check=True, cwd=d)
    return exe


def run_cases(exe: Path, cases):
    lines = []
    for case in cases:
        bits, x = case[0], case[1]
        fam = case[2] if len(case) > 2 else 0
        vals = " ".join(f"{v:.17g}" for z in x for v in (z.real, z.imag))
        lines.append(f"{bits} {len(x)} {fam} {vals}")
    out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True,
                         text=True, check=True).stdout.strip().splitlines()
    res = []
    for line in out:
        v = np.array([float(t) for t in line.split()])
        res.append(v[0::2] + 1j * v[1::2])
    return res


def test_generated_header_is_current():
    cuh, costs = gen_codelets.generate()
    gen = ROOT / "mofft_b200" / "csrc" / "generated"
    assert (gen / "codelets.cuh").read_text() == cuh
    assert (gen / "codelet_costs.h").read_text() == costs


def test_codelets_match_reference_evaluator(harness, golden_codelets):
    keys = [k[:-3] for k in golden_codelets.files if k.endswith("_in")]
    cases, wants, meta = [], [], []
    for stem in keys:
        x = golden_codelets[stem + "_in"]
        want = golden_codelets[stem + "_out"]
        radix = len(x)
        backward = "_backward_" in stem
        for bits in (32, 64):
            xin = np.conj(x) if backward else x        # bwd(x) = conj(fwd(conj(x)))
            cases.append((bits, xin))
            wants.append(want)
            meta.append((stem, bits, radix, backward))
    outs = run_cases(harness, cases)
    assert len(outs) == len(cases)
    for y, want, (stem, bits, radix, backward) in zip(outs, wants, meta):
        if backward:
            y = np.conj(y)
        tol = 64 * FLT_EPS * radix if bits == 32 else 192 * DBL_EPS * radix
        assert np.max(np.abs(y - want)) <= tol, (stem, bits)


def test_rewrite_family_codelets_match_reference_evaluator(harness, golden_codelets):
    """Every (radix, rewrite family) codelet the generator emits, both
    directions, FP32 and FP64, against the reference's evaluate_pattern
    output for that radix and pattern (rewrites.py:43-95)."""
    cases, wants, meta = [], [], []
    seen = set()
    for radix in RADICES:
        for name in gen_codelets.FAMILIES:
            if not gen_codelets.family_defined(radix, name):
                continue
            for direction in ("forward", "backward"):
                stem = f"r{radix}_{direction}_{name}"
                assert stem + "_in" in golden_codelets.files, stem
                x = golden_codelets[stem + "_in"]
                want = golden_codelets[stem + "_out"]
                backward = direction == "backward"
                for bits in (32, 64):
                    cases.append((bits, np.conj(x) if backward else x,
                                  gen_codelets.FAMILY_ID[name]))
                    wants.append(want)
                    meta.append((stem, bits, radix, backward))
                seen.add((radix, name))
    outs = run_cases(harness, cases)
    assert len(outs) == len(cases)
    for y, want, (stem, bits, radix, backward) in zip(outs, wants, meta):
        if backward:
            y = np.conj(y)
        tol = 64 * FLT_EPS * radix if bits == 32 else 192 * DBL_EPS * radix
        assert np.max(np.abs(y - want)) <= tol, (stem, bits)
    # every pattern the reference defines for each radix is covered
    assert len(seen) == sum(1 for r in RADICES for n in gen_codelets.FAMILIES
                            if gen_codelets.family_defined(r, n))
    assert (64, "like_terms_vector_reuse") in seen and (3, "like_terms") in seen


def test_bank_codelet_choice():
    """Kernel banks are chosen the way the reference's portfolio chooses
    them (portfolio.py:31-35 over model.py's ranking): every candidate of a
    radix is ranked by the cost model; bank 0 runs the best-ranked candidate
    (ties keep the hand-chosen form), bank 1 / 2 / 3 the best-ranked
    candidate carrying the like-terms / even-odd / vector-reuse rewrite, the
    bank-0 codelet where no candidate carries it."""
    assert gen_codelets.BANK_COUNT == 4
    for radix in RADICES:
        order = gen_codelets.ranked(radix)
        costs = [c.cost for c in order]
        assert costs == sorted(costs), radix
        assert sum(c.default for c in order) == 1, radix      # one hand-chosen form
        assert gen_codelets.bank_candidate(radix, 0) == order[0]
        names = {c.name for c in order}
        if radix > 2 and radix not in (3, 5, 7, 11, 13):
            # every Cooley-Tukey split is a candidate
            assert all(f"split_{a}x{radix // a}" in names
                       for a in range(2, radix) if radix % a == 0), radix
        for bank, rewrite in gen_codelets.BANK_REWRITE.items():
            chosen = gen_codelets.bank_candidate(radix, bank)
            carrying = [c for c in order if c.family and rewrite in c.family]
            assert chosen == (carrying[0] if carrying else gen_codelets.bank_candidate(radix, 0))
            fam = gen_codelets.bank_family(radix, bank)
            assert fam == (None if radix > 16 or chosen == order[0] else chosen.family)
    # instances of the rule
    assert gen_codelets.bank_family(5, 1) == "like_terms"
    assert gen_codelets.bank_family(5, 2) is None          # odd radix: no even-odd form
    assert gen_codelets.bank_family(6, 3) is None          # 6 % 4 != 0: no vector reuse
    assert gen_codelets.bank_family(16, 3) == "like_terms_vector_reuse"
    # the generated kernels run exactly these choices
    text = (ROOT / "mofft_b200" / "csrc" / "generated" / "codelets.cuh").read_text()
    for radix in (r for r in RADICES if r <= 16):
        for bank in range(1, gen_codelets.BANK_COUNT):
            fam = gen_codelets.bank_family(radix, bank)
            spec = f"struct BankDft<{radix}, {bank}> : DftFamily<{radix}, "
            if fam is None:
                assert spec not in text, (radix, bank)
            else:
                want = spec + f"{gen_codelets.FAMILY_ID[fam]}>"
                assert want in text, (radix, bank)
    report = json.loads((ROOT / "mofft_b200" / "csrc" / "generated" /
                         "codelet_portfolio.json").read_text())
    assert report["radices"]["16"]["banks"][0] == "split_4x4"
    assert report["radices"]["16"]["ranked"][0]["name"] == "split_4x4"
    # where the model prefers another form, bank 0 runs it
    assert report["radices"]["6"]["banks"][0] == "like_terms_even_odd"
    assert report["radices"]["64"]["banks"][0] == "split_16x4"
    assert "dft_fwd_6(" in text


def test_constants_correctly_rounded():
    c, s = gen_codelets.cis_turns(1, 3)
    assert c == -0.5 and s == np.sqrt(3) / 2
    for num, den in [(1, 8), (3, 16), (5, 13), (7, 64)]:
        c, s = gen_codelets.cis_turns(num, den)
        assert abs(c - np.cos(2 * np.pi * num / den)) <= 2e-16
        assert abs(s - np.sin(2 * np.pi * num / den)) <= 2e-16
