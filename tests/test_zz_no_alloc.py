"""scopi_gpu_apgd_noalloc: the APGD solve for callers that cannot allocate device memory.

Such a caller (a process whose device memory belongs to another allocator, or a loop
that must not let cudaMalloc/cudaFree synchronise the device) hands the solver device
inputs and outputs only; the solver's intermediate arrays live in a fixed array inside
the library.  This test builds one time step's contact problem, solves it through the
handle-based entry point (scopi_gpu_run) and through scopi_gpu_apgd_noalloc on device
arrays, twice in a row, and compares: the multipliers agree within the solver-tolerance
bar of the other parity tests, and the two no-allocation calls agree bit for bit (the
second call must not see the first call's leftovers).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem():
    from scopi_b200 import ScopiSolver, configs
    pa = configs.spheres_1m(side=10)
    st = configs.SETTINGS["spheres_1m"]
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    dt = st["dt"]
    s = ScopiSolver(pa, **kw).run(dt, 1)
    lam_ref = s.lagrange_multiplier()
    cont = s.current_contacts()
    s.close()
    nin = pa.nb_inactive
    na = pa.n - nin
    ci, cj = cont["i"], cont["j"]
    n = cont["nij"]
    # a-priori velocities of vap_fixed: v = v_desired (omega_desired = 0: no rotational part)
    U = pa.vd.copy()
    U[:nin] = 0.0
    au = U[ci] - U[cj]
    cvec = np.einsum("cd,cd->c", n, cont["dij"][:, None] * n + dt * au)
    rows = [[] for _ in range(na)]
    for k in range(len(ci)):
        if ci[k] >= nin:
            rows[ci[k] - nin].append(k)
        if cj[k] >= nin:
            rows[cj[k] - nin].append(k | (1 << 31))
    ptr = np.zeros(na + 1, np.int64)
    idx = []
    for p in range(na):
        r = sorted(rows[p], key=lambda e: e & 0x7FFFFFFF)
        idx.extend(r)
        ptr[p + 1] = ptr[p] + len(r)
    inc_idx = np.array(idx, dtype=np.uint32).view(np.int32)
    inv_mass = 1.0 / pa.m[nin:]
    return dict(nin=nin, na=na, ci=ci.astype(np.int32), cj=cj.astype(np.int32), n=n, c=cvec, inv_mass=inv_mass,
                ptr=ptr.astype(np.int32), idx=inc_idx, dt=dt, tol=kw["tolerance"], max_ite=kw["max_ite"],
                lam_ref=lam_ref)


def _solve(lib, P, torch):
    dev = "cuda"
    t = {k: torch.from_numpy(np.ascontiguousarray(P[k])).to(dev)
         for k in ("ci", "cj", "n", "c", "inv_mass", "ptr", "idx")}
    lam = torch.empty(len(P["ci"]), dtype=torch.float64, device=dev)
    u = torch.empty((P["na"], 3), dtype=torch.float64, device=dev)
    it = C.c_int64(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.scopi_gpu_apgd_noalloc(3, P["na"], P["nin"], len(P["ci"]), t["ci"].data_ptr(), t["cj"].data_ptr(),
                                    t["n"].data_ptr(), t["c"].data_ptr(), t["inv_mass"].data_ptr(),
                                    t["ptr"].data_ptr(), t["idx"].data_ptr(), P["dt"], 0.05, P["tol"], P["max_ite"], 1,
                                    lam.data_ptr(), u.data_ptr(), C.byref(it), stream)
    assert rc == 0, lib.scopi_gpu_last_error(None)
    torch.cuda.synchronize()
    return lam.cpu().numpy(), u.cpu().numpy(), it.value


def test_noalloc_matches_handle_path_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from scopi_b200 import _abi
    lib = _abi.load()
    P = _problem()
    assert len(P["ci"]) > 1000
    lam1, u1, it1 = _solve(lib, P, torch)
    lam2, u2, it2 = _solve(lib, P, torch)
    ref = P["lam_ref"]
    rel = np.linalg.norm(lam1 - ref) / np.linalg.norm(ref)
    assert rel <= 1e-6 and np.linalg.norm(lam1 - ref) <= 50 * P["tol"], (rel, it1)
    assert np.array_equal(lam1, lam2) and np.array_equal(u1, u2) and it1 == it2
    # u = M^-1 B^T lambda of the returned multipliers
    w = np.zeros((P["na"], 3))
    nin = P["nin"]
    for k in range(len(P["ci"])):
        if P["ci"][k] >= nin:
            w[P["ci"][k] - nin] += lam1[k] * P["n"][k]
        if P["cj"][k] >= nin:
            w[P["cj"][k] - nin] -= lam1[k] * P["n"][k]
    uexp = w * P["inv_mass"][:, None]
    assert np.linalg.norm(u1 - uexp) <= 1e-12 * max(1.0, np.linalg.norm(uexp))


def test_noalloc_rejects_sizes_beyond_its_limits():
    from scopi_b200 import _abi
    lib = _abi.load()
    it = C.c_int64(0)
    dummy = C.c_void_p(1)
    rc = lib.scopi_gpu_apgd_noalloc(3, 10, 0, 16385, dummy, dummy, dummy, dummy, dummy, dummy, dummy, 1e-3, 0.05,
                                    1e-6, 100, 1, dummy, dummy, C.byref(it), None)
    assert rc == _abi.EINVAL
    assert b"16384" in lib.scopi_gpu_last_error(None)
