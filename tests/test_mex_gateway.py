"""The MEX gateway rejects operands of the wrong size before it calls the
library (CPU, no MATLAB, no GPU).

faceted-hypersara_b200/mex/fhs_mex.c is compiled against a stand-in for the
MATLAB C API (tests/mex_stub/mex_fake.c) and a fake of the C ABI generated
from include/fhs_b200.h: an operator of 2 channels, 4 x 4 pixels, 5
visibilities and 1 block per channel, a 64-point grid; every other ABI
function counts its calls and fails with FHS_ERR_STATE.  A short operand
must end in the usage error "fhs:usage" with no library call made (the
library would otherwise write past the end of a MATLAB array); operands of
the right sizes must reach the library call.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_HAND = {
    "fhs_last_error": 'const char* fhs_last_error(void) { return "fake"; }',
    "fhs_measop_n_vis": "int64_t fhs_measop_n_vis(const fhs_measop* op, int channel) "
                        "{ (void)op; return channel >= 0 && channel < 2 ? 5 : -1; }",
    "fhs_measop_n_blocks": "int fhs_measop_n_blocks(const fhs_measop* op, int channel) "
                           "{ (void)op; return channel >= 0 && channel < 2 ? 1 : -1; }",
    "fhs_measop_grid_size": "int64_t fhs_measop_grid_size(const fhs_measop* op) { (void)op; return 64; }",
    "fhs_measop_image_size": "fhs_status fhs_measop_image_size(const fhs_measop* op, int* Ny, int* Nx, int* L) "
                             "{ (void)op; *Ny = 4; *Nx = 4; *L = 2; return FHS_OK; }",
}

_DRIVER = r"""
#include <stdio.h>
#include "mex.h"
extern int g_called;
mxArray* fake_char(const char* s);
mxArray* fake_handle(unsigned long long h);
mxArray* fake_real(size_t n);
mxArray* fake_cplx(size_t n);
mxArray* fake_cube(mwSize a, mwSize b, mwSize c);
mxArray* fake_struct(int n, const char** names, mxArray** vals);
const char* run_gateway(int nlhs, int nrhs, const mxArray** prhs);

static void report(const char* name, int nlhs, int nrhs, const mxArray** a) {
  g_called = 0;
  const char* id = run_gateway(nlhs, nrhs, a);
  printf("%s %s %d\n", name, id[0] ? id : "ok", g_called);
}

static void precond(const char* name, size_t nv2, size_t nproj, size_t ny, size_t nfx, size_t neps, size_t nsig) {
  const mxArray* a[12] = {fake_char("update_dual_data_fidelity_precond"), fake_handle(1), fake_cplx(nv2),
                          fake_cplx(nproj), fake_cplx(ny), fake_cube(4, 4, 2), fake_cplx(nfx), fake_real(neps),
                          fake_real(1), fake_real(1), fake_real(1), fake_real(nsig)};
  report(name, 7, 12, a);
}

static void dual(const char* name, size_t nv2, size_t ny, size_t nfx, size_t neps, size_t nsig) {
  const mxArray* a[8] = {fake_char("update_dual_data_fidelity"), fake_handle(1), fake_cplx(nv2), fake_cplx(ny),
                         fake_cube(4, 4, 2), fake_cplx(nfx), fake_real(neps), fake_real(nsig)};
  report(name, 6, 8, a);
}

int main(void) {
  precond("precond_ok", 10, 10, 10, 128, 2, 2);
  precond("precond_short_proj", 10, 3, 10, 128, 2, 2);
  precond("precond_empty_proj", 10, 0, 10, 128, 2, 2);
  precond("precond_short_epsilon", 10, 10, 10, 128, 1, 2);
  precond("precond_short_sigma22", 10, 10, 10, 128, 2, 1);
  precond("precond_short_fx_old", 10, 10, 10, 64, 2, 2);
  dual("dual_ok", 10, 10, 128, 2, 2);
  dual("dual_short_v2", 9, 10, 128, 2, 2);
  dual("dual_short_epsilon", 10, 10, 128, 1, 2);
  {
    const mxArray* a[4] = {fake_char("apply_direct_operator"), fake_handle(1), fake_real(1), fake_cplx(63)};
    report("direct_short_fx", 1, 4, a);
  }
  {
    const mxArray* a[4] = {fake_char("apply_adjoint_operator"), fake_handle(1), fake_real(1), fake_cplx(4)};
    report("adjoint_short_y", 1, 4, a);
  }
  {
    const mxArray* a[3] = {fake_char("HS_forward_operator_G"), fake_handle(1), fake_cube(4, 4, 1)};
    report("forward_wrong_cube", 1, 3, a);
  }
  {
    const mxArray* a[4] = {fake_char("proj_l2ball"), fake_cplx(4), fake_real(1), fake_cplx(3)};
    report("proj_short_y", 1, 4, a);
  }
  {
    const char* cn[3] = {"Ny", "Nx", "L"};
    mxArray* cv[3] = {fake_real(1), fake_real(1), fake_real(1)};
    ((double*)mxGetData(cv[0]))[0] = 4;
    ((double*)mxGetData(cv[1]))[0] = 4;
    ((double*)mxGetData(cv[2]))[0] = 2;
    const mxArray* a[8] = {fake_char("solver"), fake_handle(1), fake_char("hs"), fake_struct(3, cn, cv),
                           fake_struct(0, NULL, NULL), fake_cplx(7), fake_real(2), fake_real(0)};
    report("solver_short_y", 2, 8, a);
  }
  return 0;
}
"""


def _fake_abi(header):
    text = open(header).read()
    decls = re.findall(r"FHS_API\s+([^;(]*?)\s*\b(fhs_\w+)\s*\(([^;]*?)\)\s*;", text, flags=re.S)
    out = ['#include "fhs_b200.h"', "int g_called = 0;"]
    for ret, name, args in decls:
        ret = " ".join(ret.split())
        if name in _HAND:
            out.append(_HAND[name])
            continue
        dflt = {"fhs_status": "FHS_ERR_STATE", "const char*": '""'}.get(ret, "0")
        out.append(f"{ret} {name}({' '.join(args.split())}) {{ ++g_called; return {dflt}; }}")
    return "\n".join(out) + "\n"


def test_gateway_rejects_short_operands(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    (tmp_path / "abi_fake.c").write_text(_fake_abi(os.path.join(ROOT, "include", "fhs_b200.h")))
    (tmp_path / "driver.c").write_text(_DRIVER)
    exe = tmp_path / "gateway_check"
    r = subprocess.run([cc, "-std=c99", "-O0", "-Wall", "-Werror=implicit-function-declaration", "-I", os.path.join(ROOT, "include"),
                        "-I", os.path.join(ROOT, "tests", "mex_stub"),
                        os.path.join(ROOT, "faceted-hypersara_b200", "mex", "fhs_mex.c"),
                        os.path.join(ROOT, "tests", "mex_stub", "mex_fake.c"),
                        str(tmp_path / "abi_fake.c"), str(tmp_path / "driver.c"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    res = {ln.split()[0]: (ln.split()[1], int(ln.split()[2])) for ln in r.stdout.strip().splitlines()}
    # the right sizes reach the library (the fake fails it with FHS_ERR_STATE)
    assert res["precond_ok"] == ("fhs:error", 1), res
    assert res["dual_ok"] == ("fhs:error", 1), res
    for name, (eid, called) in res.items():
        if name.endswith("_ok"):
            continue
        assert eid == "fhs:usage" and called == 0, (name, eid, called)
