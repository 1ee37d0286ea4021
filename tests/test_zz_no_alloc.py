"""scopi_gpu_apgd_noalloc: the APGD solve for callers that cannot allocate device memory.

Such a caller (a process whose device memory belongs to another allocator, or a loop
that must not let cudaMalloc/cudaFree synchronise the device) hands the solver device
inputs and outputs only; the solver's intermediate arrays live in a fixed array inside
the library.  This test builds one time step's contact problem, solves it through the
handle-based entry point (scopi_gpu_run) and through scopi_gpu_apgd_noalloc on device
arrays, and compares: the multipliers agree within the solver-tolerance bar of the other
parity tests.  Between two solves of the same problem a different, larger problem runs
through the same fixed array, and the repeat must agree with the first solve bit for bit:
a buffer the entry point forgot to clear would carry the other problem's values into it.
Lists that would index outside their arrays are refused with SCOPI_GPU_EINVAL before the
solve reads them.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(side=10):
    from scopi_b200 import ScopiSolver, configs
    pa = configs.spheres_1m(side=side)
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


def _call(lib, P, torch, extra=0):
    """One call on device copies of P's arrays; `extra` zero entries pad inc_idx (so a
    test can lengthen inc_ptr's last entry while every read stays inside the array)."""
    dev = "cuda"
    t = {k: torch.from_numpy(np.ascontiguousarray(P[k])).to(dev)
         for k in ("ci", "cj", "n", "c", "inv_mass", "ptr")}
    t["idx"] = torch.from_numpy(np.concatenate([P["idx"], np.zeros(extra, np.int32)])).to(dev)
    lam = torch.empty(len(P["ci"]), dtype=torch.float64, device=dev)
    u = torch.empty((P["na"], 3), dtype=torch.float64, device=dev)
    it = C.c_int64(0)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.scopi_gpu_apgd_noalloc(3, P["na"], P["nin"], len(P["ci"]), t["ci"].data_ptr(), t["cj"].data_ptr(),
                                    t["n"].data_ptr(), t["c"].data_ptr(), t["inv_mass"].data_ptr(),
                                    t["ptr"].data_ptr(), t["idx"].data_ptr(), P["dt"], 0.05, P["tol"], P["max_ite"], 1,
                                    lam.data_ptr(), u.data_ptr(), C.byref(it), stream)
    torch.cuda.synchronize()
    return rc, lam.cpu().numpy(), u.cpu().numpy(), it.value


def _solve(lib, P, torch):
    rc, lam, u, it = _call(lib, P, torch)
    assert rc == 0, lib.scopi_gpu_last_error(None)
    return lam, u, it


def _close_to_handle_path(lam, P, it):
    ref = P["lam_ref"]
    rel = np.linalg.norm(lam - ref) / np.linalg.norm(ref)
    assert rel <= 1e-6 and np.linalg.norm(lam - ref) <= 50 * P["tol"], (rel, it)


def test_noalloc_matches_handle_path_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from scopi_b200 import _abi
    lib = _abi.load()
    P = _problem()
    Q = _problem(side=12)  # more contacts and bodies: fills the array past P's sizes
    assert 1000 < len(P["ci"]) < len(Q["ci"])
    lam1, u1, it1 = _solve(lib, P, torch)
    lamq, uq, itq = _solve(lib, Q, torch)
    lam2, u2, it2 = _solve(lib, P, torch)
    _close_to_handle_path(lam1, P, it1)
    _close_to_handle_path(lamq, Q, itq)
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


@pytest.mark.parametrize("fault", ["total", "decreasing", "record", "body"])
def test_noalloc_refuses_lists_outside_their_arrays(fault):
    """A malformed incidence list or contact list is refused before the solve reads it."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from scopi_b200 import _abi
    lib = _abi.load()
    P = dict(_problem())
    C_ = len(P["ci"])
    extra = 0
    if fault == "total":
        # one record more than 2 C: inc_idx is padded so the array itself is long enough
        ptr = P["ptr"].copy()
        extra = 2 * C_ + 1 - int(ptr[-1])
        ptr[-1] = 2 * C_ + 1
        P["ptr"] = ptr
    elif fault == "decreasing":
        ptr = P["ptr"].copy()
        ptr[1] = ptr[2] + 1
        P["ptr"] = ptr
    elif fault == "record":
        idx = P["idx"].copy()
        idx[0] = C_
        P["idx"] = idx
    else:
        cj = P["cj"].copy()
        cj[0] = P["nin"] + P["na"]
        P["cj"] = cj
    rc, _, _, _ = _call(lib, P, torch, extra=extra)
    assert rc == _abi.EINVAL, (rc, lib.scopi_gpu_last_error(None))
    msg = lib.scopi_gpu_last_error(None).decode()
    assert {"total": "2 * n_contacts", "decreasing": "never decrease", "record": "n_contacts",
            "body": "nb_inactive"}[fault] in msg, msg
    # the entry point still solves a well-formed problem afterwards
    Q = _problem()
    lam, _, it = _solve(lib, Q, torch)
    _close_to_handle_path(lam, Q, it)
