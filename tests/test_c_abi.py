"""The C ABI from C: include/negf_b200.h compiles as C11 and a program that
calls the library links against libnegf_b200.so, as the reference's
libnegf_c_example.c does (src/c_interface/libnegf_c_example.c links against
the reference's library).  The program runs the host-only entry points (the
DDRGF partition helpers and the reference's partition search) and its output
is checked against the oracle; calls that need a GPU are only linked."""

import ctypes
import os
import re
import shutil
import subprocess
import sys

import pytest

from conftest import ROOT
from oracle import ddrgf as o_dd

PROG = r"""
#include <stdio.h>
#include <stdlib.h>
#include "negf_b200.h"

int main(int argc, char** argv) {
  (void)argc; (void)argv;
  /* linked, not run without a GPU: the reference's C entry point */
  CCscMatrix (*wrapper)(int32_t, int32_t, int32_t, int32_t*, int32_t*, void*, int32_t, int32_t*, int32_t,
                        const char**, int32_t*, int32_t) = run_bndiag_wrapper;
  if (!wrapper) return 2;
  int32_t nr = 0, last = 0;
  for (int npl = 2; npl <= 40; ++npl)
    for (int d1 = 1; d1 <= 6; ++d1) {
      if (negf_ddrgf_get_nr_tasks(npl, d1, &nr, &last) != NEGF_SUCCESS) return 3;
      printf("T %d %d %d %d\n", npl, d1, nr, last);
    }
  int32_t lev = 0, tasks[NEGF_DDRGF_MAX_LEVELS], d1s[NEGF_DDRGF_MAX_LEVELS];
  double cost = 0.0;
  const int npls[4] = {16, 64, 128, 500};
  for (int i = 0; i < 4; ++i) {
    if (negf_ddrgf_opt_params(npls[i], 8, 2.0, 1.5, 1.0, &lev, tasks, d1s, &cost) != NEGF_SUCCESS) return 4;
    printf("O %d %d %.17g", npls[i], lev, cost);
    for (int k = 0; k < lev; ++k) printf(" %d %d", tasks[k], d1s[k]);
    printf("\n");
  }
  /* a bad argument comes back as a status and a message, not an exit */
  if (negf_ddrgf_get_nr_tasks(0, 1, &nr, &last) != NEGF_ERR_INVALID) return 5;
  if (!negf_last_error() || !negf_last_error()[0]) return 6;
  printf("version %d\n", negf_version());
  return 0;
}
"""


@pytest.fixture(scope="module")
def c_program(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    sys.path.insert(0, os.path.join(ROOT, "libnegf.jl_b200"))
    from libnegf_b200 import _lib
    libdir = os.path.dirname(_lib.LIB_PATH)
    d = tmp_path_factory.mktemp("cabi")
    src = d / "prog.c"
    src.write_text(PROG)
    exe = d / "prog"
    cmd = [cc, "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-L", libdir,
           "-lnegf_b200", "-Wl,-rpath," + libdir, "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_header_compiles_as_c11_and_links(c_program):
    assert os.path.exists(c_program)


def test_host_entry_points_from_c(c_program):
    r = subprocess.run([str(c_program)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout[-500:], r.stderr[-500:])
    n_t = n_o = 0
    for line in r.stdout.splitlines():
        f = line.split()
        if f[0] == "T":
            npl, d1, nr, last = map(int, f[1:])
            assert (nr, last) == o_dd.get_nr_tasks(npl, d1)
            n_t += 1
        elif f[0] == "O":
            npl, lev, cost = int(f[1]), int(f[2]), float(f[3])
            rest = list(map(int, f[4:]))
            lv, tasks, d1s, oc = o_dd.opt_params(npl, 2.0, 1.5, 1.0, 8)
            assert lev == lv and rest[0::2] == tasks and rest[1::2] == d1s
            assert abs(cost - oc) <= 1e-12 * oc
            n_o += 1
    assert n_t == 39 * 6 and n_o == 4
    assert "version 100" in r.stdout


LAYOUT_PROG = r"""
#include <stddef.h>
#include <stdio.h>
#include "negf_b200.h"
#define F(T, f) printf("%s %s %zu %zu\n", #T, #f, offsetof(T, f), sizeof(((T*)0)->f))
int main(void) {
  printf("size negf_solve_opts %zu\n", sizeof(negf_solve_opts));
  F(negf_solve_opts, eta); F(negf_solve_opts, mu_l); F(negf_solve_opts, mu_r); F(negf_solve_opts, kT);
  F(negf_solve_opts, want_gr); F(negf_solve_opts, want_gl); F(negf_solve_opts, want_t);
  F(negf_solve_opts, max_chunk); F(negf_solve_opts, hbm_budget_gb); F(negf_solve_opts, precision);
  F(negf_solve_opts, gemm_form); F(negf_solve_opts, gj_nb); F(negf_solve_opts, sigma_per_energy);
  F(negf_solve_opts, gj_update);
  printf("size negf_zgemm_problem %zu\n", sizeof(negf_zgemm_problem));
  F(negf_zgemm_problem, A); F(negf_zgemm_problem, B); F(negf_zgemm_problem, Cin); F(negf_zgemm_problem, C);
  F(negf_zgemm_problem, m); F(negf_zgemm_problem, n); F(negf_zgemm_problem, k); F(negf_zgemm_problem, lda);
  F(negf_zgemm_problem, ldb); F(negf_zgemm_problem, ldc); F(negf_zgemm_problem, ldcin);
  F(negf_zgemm_problem, alpha); F(negf_zgemm_problem, beta); F(negf_zgemm_problem, diag);
  printf("size CCscMatrix %zu\n", sizeof(CCscMatrix));
  F(CCscMatrix, m); F(CCscMatrix, n); F(CCscMatrix, nnz); F(CCscMatrix, colptr); F(CCscMatrix, rowval);
  F(CCscMatrix, nzval);
  return 0;
}
"""


def test_struct_layouts_match_the_bindings(tmp_path):
    """Every struct of include/negf_b200.h that a binding mirrors has the same
    fields, in the same order, at the same offsets and sizes in the Python
    ctypes layer (libnegf_b200/_lib.py), and the Julia mirror of
    negf_solve_opts in INTEGRATION.md names the same fields in the same order."""
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    sys.path.insert(0, os.path.join(ROOT, "libnegf.jl_b200"))
    from libnegf_b200 import _lib
    src = tmp_path / "layout.c"
    src.write_text(LAYOUT_PROG)
    exe = tmp_path / "layout"
    r = subprocess.run([cc, "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60).stdout.splitlines()
    c_fields, c_size = {}, {}
    for line in out:
        f = line.split()
        if f[0] == "size":
            c_size[f[1]] = int(f[2])
        else:
            c_fields.setdefault(f[0], []).append((f[1], int(f[2]), int(f[3])))
    mirrors = {"negf_solve_opts": _lib.SolveOpts, "negf_zgemm_problem": _lib.ZGemmProblem,
               "CCscMatrix": _lib.CCscMatrix}
    for cname, py in mirrors.items():
        assert ctypes.sizeof(py) == c_size[cname], cname
        py_fields = [(name, getattr(py, name).offset, getattr(py, name).size) for name, _ in py._fields_]
        assert py_fields == c_fields[cname], cname
    # the Julia struct in INTEGRATION.md
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    body = re.search(r"struct NegfOpts\n(.*?)\nend", text, re.S).group(1)
    jl_names = re.findall(r"(\w+)::", body)
    assert jl_names == [f[0] for f in c_fields["negf_solve_opts"]]
