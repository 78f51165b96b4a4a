"""Test helpers: run md_* entry points on device copies of numpy arrays (via torch
CUDA tensors) and the matching oracle functions on host copies."""
import ctypes as C

import numpy as np

import oracle
import rfdem

ID_NP = rfdem.ID_NP


def dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64).copy()).cuda()
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).cuda()
    return torch.from_numpy(a.copy()).cuda()


def host(t, dtype):
    torch_sync(t)
    a = t.cpu().numpy()
    return a.view(dtype) if a.dtype != np.dtype(dtype) else a


def torch_sync(t):
    import torch
    torch.cuda.synchronize()


def grid_args(task):
    return task.C.a, task.C._1d_a, task.C.Nr, int(task.C.N)


# --- GPU (md_*) -----------------------------------------------------------------
def gpu_cells(torch, task, R):
    N = R.size // 3
    CN = int(task.C.N)
    dR = dev(torch, R)
    CI = torch.zeros(N, dtype=torch.int64, device="cuda")
    CIs = torch.zeros(2 * N, dtype=torch.int64, device="cuda")
    pnC = torch.zeros(2 * CN, dtype=torch.int64, device="cuda")
    sb = rfdem.lib.md_CellDistributionScratchBytes(N, CN)
    scratch = torch.zeros(sb, dtype=torch.uint8, device="cuda")
    st = rfdem.lib.md_CellDistribution(dR.data_ptr(), N, CI.data_ptr(), CIs.data_ptr(), pnC.data_ptr(), CN,
                                       task.C._1d_a, task.C.Nr, scratch.data_ptr(), sb, None)
    return st, host(CI, ID_NP), host(CIs, ID_NP), host(pnC, ID_NP)


def gpu_list_construct(torch, task, R, CIs, pnC):
    N, K = R.size // 3, int(task.K)
    a, inv_a, Nr, CN = grid_args(task)
    dIL = torch.zeros(N * K, dtype=torch.int64, device="cuda")
    keep = [dev(torch, R), dev(torch, CIs), dev(torch, pnC)]       # alive until the kernel has run
    st = rfdem.lib.md_InteractionListConstruct(keep[0].data_ptr(), N, keep[1].data_ptr(), keep[2].data_ptr(),
                                               dIL.data_ptr(), K, a, inv_a, task.aacut, Nr, CN, None)
    out = host(dIL, ID_NP)
    del keep
    return st, out


def gpu_reconstruct(torch, task, R, CIs, pnC, IL, ty):
    N, K = R.size // 3, int(task.K)
    a, inv_a, Nr, CN = grid_args(task)
    dIL, dT = dev(torch, IL), dev(torch, ty)
    keep = [dev(torch, R), dev(torch, CIs), dev(torch, pnC)]       # alive until the kernel has run
    st = rfdem.lib.md_InteractionListReConstructBPM(keep[0].data_ptr(), N, keep[1].data_ptr(), keep[2].data_ptr(),
                                                    dIL.data_ptr(), dT.data_ptr(), K, a, inv_a, task.aacut, Nr, CN,
                                                    None)
    out = host(dIL, ID_NP), host(dT, np.uint8)
    del keep
    return (st,) + out


def zeros_state(N, K):
    return {k: np.zeros(3 * N * K, np.float32) for k in ["Rij", "Oijt", "Fijn", "Fijt", "Mijn", "Mijt", "Mijadd"]}


def gpu_bonds_delete(torch, task, R, IL, ty, iL, S, aa_create, aa_far, do_bonds=True, do_delete=True):
    N, K = R.size // 3, int(task.K)
    dR = dev(torch, R)
    dIL, dT, diL = dev(torch, IL), dev(torch, ty), dev(torch, iL)
    dS = {k: dev(torch, v) for k, v in S.items()}
    order = ["Rij", "Oijt", "Fijn", "Fijt", "Mijn", "Mijt", "Mijadd"]
    if do_bonds:
        rfdem.check(rfdem.lib.md_ConstructBoundInteractions(dR.data_ptr(), dR.data_ptr(), dR.data_ptr(), dIL.data_ptr(),
                                                            dT.data_ptr(), diL.data_ptr(),
                                                            *[dS[k].data_ptr() for k in order], N, K, aa_create,
                                                            task.Po.b_r, None))
    if do_delete:
        rfdem.check(rfdem.lib.md_DeleteFarLinks(dR.data_ptr(), N, dIL.data_ptr(), dT.data_ptr(), diL.data_ptr(),
                                                *[dS[k].data_ptr() for k in order], K, aa_far, None))
    return host(dIL, ID_NP), host(dT, np.uint8), host(diL, np.float32), {k: host(v, np.float32) for k, v in dS.items()}


def bond_params(task):
    P = task.Po
    f = lambda x: float(np.float32(x))
    return [f(P.dt), f(P.m_E), f(P.m_G), f(P.b_r), f(P.m_Ec), f(P.m_Gc)]


def contact_params(task):
    P = task.Po
    f = lambda x: float(np.float32(x))
    return [f(P.dt), f(P.hm_E), f(P.hm_G), f(P.p_A), f(P.p_mu), f(P.p_mur), f(P.p_m), f(P.p_r)]


def gpu_forces(torch, task, R, V, W, IL, ty, iL, S):
    N, K = R.size // 3, int(task.K)
    d = {k: dev(torch, v) for k, v in dict(R=R, V=V, W=W, IL=IL, ty=ty, iL=iL, **S).items()}
    F = torch.zeros(3 * N, dtype=torch.float32, device="cuda")
    M = torch.zeros(3 * N, dtype=torch.float32, device="cuda")
    rfdem.check(rfdem.lib.md_CalculateForcesDEM_22(d["R"].data_ptr(), d["V"].data_ptr(), d["W"].data_ptr(),
                                                   d["IL"].data_ptr(), d["ty"].data_ptr(), d["iL"].data_ptr(),
                                                   d["Rij"].data_ptr(), d["Oijt"].data_ptr(), d["Mijn"].data_ptr(),
                                                   d["Mijt"].data_ptr(), F.data_ptr(), M.data_ptr(), N, K,
                                                   *bond_params(task), None))
    rfdem.check(rfdem.lib.md_CalculateForcesDEM_21(d["R"].data_ptr(), d["V"].data_ptr(), d["W"].data_ptr(),
                                                   d["IL"].data_ptr(), d["ty"].data_ptr(), d["iL"].data_ptr(),
                                                   d["Rij"].data_ptr(), d["Oijt"].data_ptr(), F.data_ptr(),
                                                   M.data_ptr(), N, K, *contact_params(task), None))
    out = dict(F=host(F, np.float32), M=host(M, np.float32), ty=host(d["ty"], np.uint8))
    for k in ["Rij", "Oijt", "Mijn", "Mijt"]:
        out[k] = host(d[k], np.float32)
    return out


def clone(task):
    return rfdem.Task.from_buffer_copy(task)


# --- oracle -----------------------------------------------------------------------
def p(a):
    return a.ctypes.data


def oracle_cells(task, R):
    L = oracle.load()
    N = R.size // 3
    CN = int(task.C.N)
    CI, CIs, pnC = np.zeros(N, np.uint64), np.zeros(2 * N, np.uint64), np.zeros(2 * CN, np.uint64)
    st = L.rfo_cell_distribution_f(p(R), N, p(CI), p(CIs), p(pnC), CN, task.C._1d_a, task.C.Nr)
    return st, CI, CIs, pnC


def oracle_list_construct(task, R, CIs, pnC):
    L = oracle.load()
    N, K = R.size // 3, int(task.K)
    a, inv_a, Nr, CN = grid_args(task)
    IL = np.zeros(N * K, np.uint64)
    st = L.rfo_construct_list_f(p(R), N, p(CIs), p(pnC), p(IL), K, a, inv_a, task.aacut, Nr, CN)
    return st, IL


def oracle_reconstruct(task, R, CIs, pnC, IL, ty):
    L = oracle.load()
    N, K = R.size // 3, int(task.K)
    a, inv_a, Nr, CN = grid_args(task)
    IL, ty = IL.copy(), ty.copy()
    st = L.rfo_reconstruct_bpm_f(p(R), N, p(CIs), p(pnC), p(IL), p(ty), K, a, inv_a, task.aacut, Nr, CN)
    return st, IL, ty


def oracle_bonds_delete(task, R, IL, ty, iL, S, aa_create, aa_far, do_bonds=True, do_delete=True):
    L = oracle.load()
    N, K = R.size // 3, int(task.K)
    IL, ty, iL = IL.copy(), ty.copy(), iL.copy()
    S = {k: v.copy() for k, v in S.items()}
    if do_bonds:
        L.rfo_construct_bonds_f(p(R), N, p(IL), p(ty), p(iL), p(S["Rij"]), p(S["Oijt"]), p(S["Mijn"]), p(S["Mijt"]),
                                K, aa_create)
    if do_delete:
        L.rfo_delete_far_links_f(p(R), N, p(IL), p(ty), p(S["Rij"]), p(S["Oijt"]), p(S["Mijn"]), p(S["Mijt"]), K,
                                 aa_far)
    return IL, ty, iL, S


def oracle_forces(task, R, V, W, IL, ty, iL, S):
    L = oracle.load()
    N, K = R.size // 3, int(task.K)
    ty = ty.copy()
    S = {k: v.copy() for k, v in S.items()}
    F, M = np.zeros(3 * N, np.float32), np.zeros(3 * N, np.float32)
    L.rfo_forces_22_f(p(R), p(V), p(W), p(IL), p(ty), p(iL), p(S["Rij"]), p(S["Oijt"]), p(S["Mijn"]), p(S["Mijt"]),
                      p(F), p(M), N, K, *bond_params(task), None)
    L.rfo_forces_21_f(p(R), p(V), p(W), p(IL), p(ty), p(S["Oijt"]), p(F), p(M), N, K, *contact_params(task))
    out = dict(F=F, M=M, ty=ty)
    for k in ["Rij", "Oijt", "Mijn", "Mijt"]:
        out[k] = S[k]
    return out


def oracle_state_after(task, R0, steps):
    """Oracle FP32 state after `steps` explicit steps (reference layout)."""
    t = clone(task)
    n, st, curve, status = oracle.run_f(t, R0, steps)
    return t, st
