"""The C ABI (include/nociwick.h) without a GPU: exports, struct layouts, error paths."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import nociwick
from nociwick import lib as L
from nociwick.synthetic import NW_DET_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nociwick.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"NW_API\s+(?:const\s+)?\w+\*?\s+(nw_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = header_functions()
    assert len(names) >= 12
    lib = ctypes.CDLL(nociwick.LIB_PATH)
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(L.EXPORTED)


def test_struct_layouts_match_bindings(tmp_path):
    probe = tmp_path / "probe.c"
    probe.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "nociwick.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(nw_det), offsetof(nw_det, rank_a), offsetof(nw_det, idx_a),
         offsetof(nw_det, rank_b), offsetof(nw_det, idx_b), offsetof(nw_det, phase), sizeof(nw_system));
  printf("%zu %zu %zu %zu %zu\n", sizeof(nw_refs), sizeof(nw_opts), sizeof(nw_info),
         offsetof(nw_system, s), offsetof(nw_refs, c_alpha));
  printf("%zu %zu %zu %zu %zu\n", sizeof(nw_qmc_opts), offsetof(nw_qmc_opts, ncycles), offsetof(nw_qmc_opts, seed),
         sizeof(nw_qmc_report), offsetof(nw_qmc_report, nocc));
  printf("%zu %zu %zu %zu %zu\n", sizeof(nw_pt2_projection), sizeof(nw_gmres_opts), offsetof(nw_gmres_opts, res_tol),
         offsetof(nw_gmres_opts, preconditioner), sizeof(nw_gmres_info));
  printf("%zu %zu %zu %zu\n", sizeof(nw_mlp_opts), offsetof(nw_mlp_opts, seed), sizeof(nw_mlp_report),
         offsetof(nw_mlp_report, steps));
  printf("%zu %zu %zu\n", sizeof(nw_tune_report), offsetof(nw_tune_report, trials), offsetof(nw_tune_report, default_ms));
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(nw_system_cd), offsetof(nw_system_cd, naux), offsetof(nw_system_cd, enuc),
         offsetof(nw_system_cd, chol), sizeof(nw_exc_cache), offsetof(nw_exc_cache, beta));
  return 0;
}
''')
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(probe), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    v = [int(x) for x in out]
    f = NW_DET_DTYPE.fields
    assert v[:6] == [NW_DET_DTYPE.itemsize, f["rank_a"][1], f["idx_a"][1], f["rank_b"][1], f["idx_b"][1],
                     f["phase"][1]]
    assert v[6] == ctypes.sizeof(L.NwSystem)
    assert v[7:10] == [ctypes.sizeof(L.NwRefs), ctypes.sizeof(L.NwOpts), ctypes.sizeof(L.NwInfo)]
    assert v[10] == L.NwSystem.s.offset and v[11] == L.NwRefs.c_alpha.offset
    assert v[12:17] == [ctypes.sizeof(L.NwQmcOpts), L.NwQmcOpts.ncycles.offset, L.NwQmcOpts.seed.offset,
                        ctypes.sizeof(L.NwQmcReport), L.NwQmcReport.nocc.offset]
    assert v[17:22] == [ctypes.sizeof(L.NwPt2Projection), ctypes.sizeof(L.NwGmresOpts), L.NwGmresOpts.res_tol.offset,
                        L.NwGmresOpts.preconditioner.offset, ctypes.sizeof(L.NwGmresInfo)]
    assert v[22:26] == [ctypes.sizeof(L.NwMlpOpts), L.NwMlpOpts.seed.offset, ctypes.sizeof(L.NwMlpReport),
                        L.NwMlpReport.steps.offset]
    assert v[26:29] == [ctypes.sizeof(L.NwTuneReport), L.NwTuneReport.trials.offset, L.NwTuneReport.default_ms.offset]
    assert v[29:33] == [ctypes.sizeof(L.NwSystemCd), L.NwSystemCd.naux.offset, L.NwSystemCd.enuc.offset,
                        L.NwSystemCd.chol.offset]
    assert v[33:35] == [L.NW_EXC_CACHE_DTYPE.itemsize, L.NW_EXC_CACHE_DTYPE.fields["rank_b"][1]]


def test_header_compiles_as_cxx(tmp_path):
    src = tmp_path / "probe.cpp"
    src.write_text('#include "nociwick.h"\nint main() { return nw_status_string(NW_OK) ? 0 : 1; }\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                    str(src)], check=True)


def test_status_strings_and_argument_errors():
    lib = L.load()
    assert lib.nw_status_string(0) == b"ok"
    assert lib.nw_status_string(6) == b"no CUDA device"
    out = ctypes.c_void_p()
    assert lib.nw_ctx_create(None, None, None, ctypes.byref(out)) == 1
    assert lib.nw_ctx_destroy(None) == 0
    assert lib.nw_build_intermediates(None) == 1
    assert lib.nw_eval_hs_pairs(None, None, 0, None, None) == 1


def test_invalid_system_rejected_before_device_use():
    from nociwick import synthetic as sy
    s = sy.make_system(6, 2, 2, 2, 10, seed=1)
    h = s.h.copy()
    h[0, 0] = np.nan
    with pytest.raises(L.NwError) as e:
        nociwick.WicksShared(s.s, h, s.eri, s.enuc, s.refs)
    assert e.value.status == 1


def test_no_device_reported_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from nociwick import synthetic as sy
    s = sy.make_system(6, 2, 2, 2, 10, seed=1)
    with pytest.raises(L.NwError) as e:
        nociwick.WicksShared(s.s, s.h, s.eri, s.enuc, s.refs)
    assert e.value.status == 6


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError):
        L.load(str(tmp_path / "absent.so"))


def test_cxx_host_interface_compiles_and_links(tmp_path):
    """The header-only C++ mirror of the reference interface builds against the library."""
    src = tmp_path / "use.cpp"
    src.write_text(r'''
#include "wicks.hpp"
int main() {
  nociwick::AoData ao;
  nociwick::References refs;
  try {
    auto w = nociwick::build_wicks_shared(ao, refs, 1e-8);
    (void)w;
  } catch (const nociwick::Error& e) {
    return e.status == NW_ERR_INVALID ? 0 : 1;
  }
  return 2;
}
''')
    exe = tmp_path / "use"
    libdir = os.path.dirname(nociwick.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "noci-rs_b200", "host"),
                    str(src), "-L", libdir, "-lnociwick", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    # empty inputs are rejected with NW_ERR_INVALID before any device use
    assert subprocess.run([str(exe)]).returncode == 0
