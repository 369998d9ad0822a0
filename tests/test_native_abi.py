"""The C ABI library without a GPU: it loads, exports every function that
include/tbpm_b200.h declares, computes host-only quantities, and refuses to
run device work when no GPU is present (no CPU fallback)."""

import os
import re

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200 import _native as nat
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "tbpm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tbpm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    lib = nat.load_library()
    declared = _declared_functions()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(nat.EXPORTED_SYMBOLS) == declared
    assert lib.tbpm_version() == 1


def test_fermi_coefficients_host_only_match_oracle():
    beta = 9.0 / (tb.KB * 300)
    for mu, omf in ((0.0, False), (0.0, True), (0.02, False)):
        a = nat.fermi_cheb_coef(2**15, beta, mu, omf, 1e-12)
        b = oracle.fermi_cheb_coef(2**15, beta, mu, omf, 1e-12)
        assert a.size == b.size
        assert np.max(np.abs(a - b)) < 1e-14
    with pytest.raises(ValueError):
        nat.fermi_cheb_coef(1000, beta, 0.0, False, 1e-12)  # not a power of two


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the behaviour without a GPU")
def test_no_gpu_fails_loudly():
    with pytest.raises(nat.TbpmError):
        nat.Context(0)
    from tbplas_b200.fortran import f2py
    s = tb.make_graphene_sample(4, 4)
    h = s.build_ham_csr()
    nat._contexts.clear()
    with pytest.raises(nat.TbpmError):
        f2py.tbpm_dos([1.0, 0.1, 0.01], h.indptr, h.indices, h.data, 1, 4, 1, "", 0, 128, 1e-9)


def test_f2py_argument_validation_happens_on_host():
    from tbplas_b200.fortran import f2py
    with pytest.raises(ValueError):
        f2py._csr(np.array([0, 2 ** 40]), np.array([0]), np.array([1.0]))
    with pytest.raises(ValueError):
        f2py._csr(np.array([0]), np.array([]), np.array([]))
    with pytest.raises(ValueError):
        f2py.set_backend(precision="fp16")
    with pytest.raises(ValueError):
        f2py.set_backend(nonsense=1)


def test_device_sample_interface_without_device_work():
    """DeviceSample exposes the Sample interface the Solver and Analyzer read;
    without a GPU its assembly raises instead of building on the host."""
    s = tb.make_graphene_device_sample(4, 3, rescale=9.0)
    ref = tb.LatticeSample((4, 3))
    assert s.num_orb == ref.num_orb == 24
    assert s.area_unit_cell == ref.area_unit_cell
    assert s.volume_unit_cell == ref.volume_unit_cell
    assert s.nr_orbitals == 2 and s.extended == 1.0
    assert s.rescale == 9.0 and s.energy_range == 18.0
    h = s.build_ham_csr()
    assert hasattr(h.indptr, "make_resident") and h.shape == (24, 24)
    ip, ix, hop, dx, dy = s.build_ham_dxy()
    assert hasattr(ip, "make_resident") and ix is None and dx is None
    with pytest.raises(ValueError):
        tb.DeviceSample(np.eye(3), None, [[0, 0, 0]], [0.0, 1.0], [[1, 0, 0, 0, 0]], [-1.0],
                        (3, 1, 1))
    with pytest.raises(ValueError):
        tb.make_graphene_device_sample(4, 3, gauge=5)
    if not _gpu_present():
        nat._contexts.clear()
        with pytest.raises(nat.TbpmError):
            s.download_ham_csr()


def test_checkpoint_fingerprint_tracks_every_input(tmp_path):
    from tbplas_b200 import checkpoint as ck
    from tbplas_b200.fortran import f2py
    s = tb.make_graphene_sample(4, 4, disorder=0.5, rescale=9.0, seed=1)
    h = s.build_ham_csr()
    be = f2py.get_backend()
    base = ck.fingerprint([0.5, 0.2, 0.1], h.indptr, h.indices, h.data, 1, 10, 2, 0, be)
    assert base == ck.fingerprint([0.5, 0.2, 0.1], h.indptr, h.indices, h.data, 1, 10, 2, 0, be)
    other = h.data.copy()
    other[3] += 1e-12
    variants = [
        ck.fingerprint([0.5, 0.2, 0.1], h.indptr, h.indices, other, 1, 10, 2, 0, be),
        ck.fingerprint([0.5, 0.2, 0.11], h.indptr, h.indices, h.data, 1, 10, 2, 0, be),
        ck.fingerprint([0.5, 0.2, 0.1], h.indptr, h.indices, h.data, 2, 10, 2, 0, be),
        ck.fingerprint([0.5, 0.2, 0.1], h.indptr, h.indices, h.data, 1, 11, 2, 0, be),
        ck.fingerprint([0.5, 0.2, 0.1], h.indptr, h.indices, h.data, 1, 10, 2, 0,
                       dict(be, precision="fp32")),
    ]
    assert len(set(variants + [base])) == len(variants) + 1
    path = str(tmp_path / "c.npz")
    ck._save(path, fingerprint=np.array(base), s0=np.array(3))
    assert int(ck._load(path, base)["s0"]) == 3
    assert ck._load(path, variants[0]) is None
    (tmp_path / "bad.npz").write_bytes(b"not a zip")
    assert ck._load(str(tmp_path / "bad.npz"), base) is None


def test_header_is_plain_c():
    """include/tbpm_b200.h is the drop-in boundary for C FFIs (cgo, ctypes,
    JNI stubs): it must compile as C99 on its own, with no C++ types."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    hdr = os.path.join(root, "include", "tbpm_b200.h")
    r = subprocess.run([cc, "-x", "c", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", hdr],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_program_links_and_calls_host_entry_points(tmp_path):
    """A plain C caller (as a cgo or JNI stub would be) links against
    libtbpm_b200.so and calls the host-only entry points; its Fermi
    coefficients equal the Python binding's."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "caller.c"
    src.write_text(r"""
#include <stdio.h>
#include <stdlib.h>
#include "tbpm_b200.h"
int main(void) {
  int n = 0, rc;
  double* c = (double*)malloc(sizeof(double) * 32768);
  printf("%d\n", tbpm_version());
  rc = tbpm_fermi_cheb_coef(32768, 9.0 / (8.617333262e-5 * 300.0), 0.0, 1, 1e-12, c, &n);
  printf("%d %d %.17g %.17g\n", rc, n, c[0], c[n - 1]);
  rc = tbpm_fermi_cheb_coef(1000, 1.0, 0.0, 0, 1e-12, c, &n);
  printf("%d\n", rc != 0);
  free(c);
  return 0;
}
""")
    exe = tmp_path / "caller"
    lib_dir = os.path.join(root, "tbplas_b200")
    r = subprocess.run([cc, "-std=c99", "-O1", str(src), "-I", os.path.join(root, "include"),
                        "-L", lib_dir, "-ltbpm_b200", "-Wl,-rpath," + lib_dir, "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.split("\n")
    assert int(lines[0]) > 0
    rc, n, c0, cl = lines[1].split()
    ref = nat.fermi_cheb_coef(2**15, 9.0 / (8.617333262e-5 * 300.0), 0.0, True, 1e-12)
    assert int(rc) == 0 and int(n) == ref.size
    assert float(c0) == ref[0] and float(cl) == ref[-1]
    assert lines[2] == "1"  # a size that is not a power of two is rejected


def test_status_codes_map_to_python_errors():
    """TBPM_ERR_NAN becomes NanError, which callers that catch the reference's
    broken-norm failure (NormError) also catch."""
    with pytest.raises(nat.NanError) as e:
        nat.raise_for(nat.TBPM_ERR_NAN, "tbpm_dos: the wave function norm is NaN")
    assert isinstance(e.value, nat.NormError) and e.value.code == nat.TBPM_ERR_NAN
    with pytest.raises(nat.NormError) as e:
        nat.raise_for(nat.TBPM_ERR_NORM, "broken")
    assert not isinstance(e.value, nat.NanError)
    with pytest.raises(ValueError):
        nat.raise_for(nat.TBPM_ERR_ARG, "bad")


def test_checkpointed_run_rejects_zero_steps(tmp_path):
    from tbplas_b200.checkpoint import dos_checkpointed
    ip = np.array([0, 1, 2], dtype=np.int32)
    ix = np.array([1, 0], dtype=np.int32)
    hv = np.ones(2, dtype=np.complex128)
    with pytest.raises(ValueError, match="n_timestep"):
        dos_checkpointed([1.0, 0.5, 0.1], ip, ix, hv, 1337, 0, 1, 0, 128, 1e-9,
                         str(tmp_path / "c.npz"))
