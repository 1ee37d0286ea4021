"""C ABI checks that need no GPU: the library builds for sm_100a, loads, and exports
every function include/scopi_gpu.h declares; the Python mirror exposes the reference
parameter names."""
import os
import re
import shutil

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "scopi_gpu.h")).read()
    return sorted(set(re.findall(r"\b(scopi_gpu_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from scopi_b200 import _abi
    if not os.path.exists(_abi.LIB_PATH):
        if shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"):
            pytest.skip("nvcc unavailable")
        from scopi_b200 import build
        build.build()
    return _abi.load()


def test_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/scopi_gpu.h but not exported"


def test_python_binding_covers_header():
    from scopi_b200 import _abi
    assert set(declared_symbols()) == set(_abi.EXPORTED)


def test_default_params_match_reference(lib):
    import ctypes as C
    from scopi_b200 import _abi
    p = _abi.Params()
    lib.scopi_gpu_default_params(C.byref(p), 3)
    # apgd.hpp:120-123, contact_kdtree.hpp:229-237, property.hpp:72,125-127
    assert (p.alpha, p.max_ite, p.tolerance, p.dynamic_descent) == (0.05, 10000, 1e-7, 1)
    assert (p.dmax, p.kd_tree_radius) == (2.0, 17.0)
    assert (p.mu, p.gamma, p.gamma_min, p.gamma_tol) == (0.1, 0.0, -2.0, 1e-6)


def test_create_without_gpu_fails_cleanly(lib):
    import ctypes as C
    import torch
    from scopi_b200 import _abi
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = _abi.Params()
    lib.scopi_gpu_default_params(C.byref(p), 2)
    h = C.c_void_p()
    rc = lib.scopi_gpu_create(C.byref(p), C.byref(h))
    assert rc == _abi.ECUDA and not h.value
    assert b"CUDA" in lib.scopi_gpu_last_error(None)


def test_set_state_without_handle_is_refused(lib):
    # host-side argument checks only: no CUDA call is reached
    from scopi_b200 import _abi
    assert lib.scopi_gpu_set_state(None, None) == _abi.EINVAL


def test_solver_raises_without_library(tmp_path):
    from scopi_b200 import _abi
    with pytest.raises(OSError):
        _abi._lib, saved = None, _abi._lib
        try:
            _abi.load(str(tmp_path / "missing.so"))
        finally:
            _abi._lib = saved


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of scopi_gpu_params / _particles / _stats have the C layout (size and
    the offsets of the fields added last), checked against the header compiled by gcc."""
    import ctypes as C
    import subprocess
    from scopi_b200 import _abi
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "scopi_gpu.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(scopi_gpu_params), '
                   'offsetof(scopi_gpu_params, fixed_point_tol), offsetof(scopi_gpu_params, box_lower), '
                   'offsetof(scopi_gpu_params, periodic), sizeof(scopi_gpu_particles), '
                   'offsetof(scopi_gpu_particles, worm), sizeof(scopi_gpu_stats)); return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(_abi.Params), _abi.Params.fixed_point_tol.offset, _abi.Params.box_lower.offset,
            _abi.Params.periodic.offset, C.sizeof(_abi.ParticlesC), _abi.ParticlesC.worm.offset, C.sizeof(_abi.Stats)]
    assert got == want


def test_default_params_have_no_box(lib):
    import ctypes as C
    from scopi_b200 import _abi
    from scopi_b200.solver import _set_param
    p = _abi.Params()
    lib.scopi_gpu_default_params(C.byref(p), 3)
    assert list(p.periodic) == [0, 0, 0] and list(p.box_lower) == [0.0] * 3
    assert (p.fixed_point_tol, p.fixed_point_max_iter) == (1e-6, 1000)
    _set_param(p, "box_upper", (4.0, 2.0))
    _set_param(p, "periodic", (1, 0))
    assert list(p.box_upper) == [4.0, 2.0, 0.0] and list(p.periodic) == [1, 0, 0]


def test_worm_indices_in_the_container():
    from scopi_b200.container import Particles, Property
    p = Particles(2)
    p.add_sphere((0.0, 5.0), 0.5, Property())
    p.add_worm([(1.0, 0.0), (3.0, 0.0), (5.0, 0.0)], 1.0, Property(desired_velocity=(1.0, 0.0)))
    p.add_worm([(1.0, 3.0), (3.0, 3.0)], 1.0, Property())
    pa = p.finalize()
    assert pa.worm.dtype.name == "int32" and pa.worm.tolist() == [-1, 0, 0, 0, 1, 1]
    assert pa.radius.tolist() == [0.5, 1.0, 1.0, 1.0, 1.0, 1.0]
    assert pa.vd[1:4, 0].tolist() == [1.0, 1.0, 1.0]
    assert pa.copy().worm.tolist() == pa.worm.tolist()
