"""The reference's own known-answer checks (cases.c) run against the
compiled oracle (oracle/_ref): they pin the project-written single-rank MPI
and FFTW shims the oracle is built on.

Each case prints a line only where its check fails, so a clean run prints
its banner and nothing else:
* case 1 / case 8 (2nd / 4th order): the projected field has zero discrete
  divergence, |div| <= 1e-10 (cases.c:486, 2546), and the pressure solves
  the discrete Poisson equation, |L p - div| <= 1e-10 (cases.c:501, 2561);
  failures print "ix=.. iy=.. iz=.. div=" / "err=";
* case 14: the restart-file write / read round trip is exact to DBL_EPSILON
  (cases.c:4271); failures print three numbers per line;
* case 15: get_xy_moment agrees with get_xy_corr, |mom1| < 1e-13 and
  |mom2 - corr| < 1e-13 (cases.c:4397-4398), through check(), which aborts;
* case 16: Parseval -- the x and y cospectra sum to the correlation and the
  quadrature spectra to zero within 1e-15 (cases.c:4683-4686); failures
  print "k d d d d".

Every case runs in a child process whose working directory is a temporary
folder (case 14 writes tmp.dat there), so that its C stdout can be read.
"""
import os
import re
import subprocess
import sys

import pytest

ORACLE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle")

NUM = r"[+-]?\d\.\d+e[+-]\d+"
VIOLATION = {
    1: re.compile(r"^ix=\d+ iy=\d+ iz=\d+ (div|err)="),
    8: re.compile(r"^ix=\d+ iy=\d+ iz=\d+ (div|err)="),
    14: re.compile(rf"^{NUM} {NUM} {NUM}$"),
    15: None,
    16: re.compile(rf"^\d+ {NUM} {NUM} {NUM} {NUM}$"),
}
BANNER = {1: "Check 2nd-order pressure Poisson solver", 8: "Check 4th-order pressure Poisson solver",
          14: "Reading temporary file", 15: "Check consistency of get_xy_moment()", 16: "Testing get_xy_spec()"}


def run_case(which, nx, ny, nz, cwd):
    code = ("import sys; sys.path.insert(0, %r); import ref; "
            "rc = ref.lib().ref_case(%d, %d, %d, %d, 3); sys.stdout.flush(); print('RC', rc)"
            % (ORACLE, which, nx, ny, nz))
    r = subprocess.run([sys.executable, "-c", code], cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=300)
    return r.returncode, r.stdout


@pytest.mark.parametrize("nx,ny,nz", [(32, 24, 16), (48, 40, 20)])
@pytest.mark.parametrize("which", [1, 8, 14, 15, 16])
def test_reference_case_passes(ref, tmp_path, which, nx, ny, nz):
    rc, out = run_case(which, nx, ny, nz, str(tmp_path))
    assert rc == 0, out
    lines = out.splitlines()
    assert "RC 0" in lines, out          # ref_case returns -1 when check() aborted
    assert BANNER[which] in lines, out
    pat = VIOLATION[which]
    if pat is not None:
        bad = [ln for ln in lines if pat.match(ln)]
        assert not bad, bad[:5]
    if which in (1, 8):
        # the projected field's mean blowing velocity at both walls: the case
        # prints it before and after the projection; it must stay finite
        avg = [ln for ln in lines if ln.startswith("avg_bot=")]
        assert len(avg) == 2, out
    assert not os.path.exists(tmp_path / "tmp.dat")   # case 14 removes its file
