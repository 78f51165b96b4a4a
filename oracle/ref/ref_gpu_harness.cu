// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// Harness that runs the RockFit-DEM reference's OWN kernels and host step
// functions (compiled from its sources, unmodified, for sm_100a) on host arrays,
// so the tests can compare the engine with the reference on identical inputs.
// Built by oracle/build.py into oracle/_ref/libmdref_gpu.so with oracle/ref/ids32.h
// forced in (the reference's 4-byte ids). Only tests load it.
//
// Every device buffer is allocated with slack so the reference's known reads
// past the end stay inside an allocation:
//   IL[(N)*K] is read one slot past the last row (md_boundinteractions_construct.cu:101-102);
//   CIs[2N] can be read when the last cell run is extended (md_calculate_cell.cu:72).
// The tests keep particles away from the cell-grid border, where the reference
// would index pnC outside the grid (md_interaction_list_reconstructbpm.cu:99-118).

#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <vector>
#include "md.h"
#include "md_data_types.h"
#include "../../include/rockfit_b200.h"

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
    fprintf(stderr, "ref harness: %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); return -1; } } while (0)

namespace {
const size_t SLACK = 4096;   // elements of slack after every array

template <class T> T* dalloc(size_t n, int fill = 0) {
    T* p = nullptr;
    if (cudaMalloc((void**)&p, (n + SLACK) * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemset(p, fill, (n + SLACK) * sizeof(T));
    return p;
}
template <class T> int up(T* d, const T* h, size_t n) {
    if (!h) return 0;
    return cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : -1;
}
template <class T> int down(T* h, const T* d, size_t n) {
    if (!h) return 0;
    return cudaMemcpy(h, d, n * sizeof(T), cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : -1;
}

struct Dev {
    particle_data P{};
    cell_data C{};
    additional_data A;
    sample_data S{};
    interaction_list_data IL{};
    uint32_t N = 0, K = 0;

    int alloc(uint32_t n, uint32_t k, uint32_t cn) {
        N = n; K = k;
        P.N = n;
        P.d_R = dalloc<float>(3 * (size_t)n); P.d_V = dalloc<float>(3 * (size_t)n);
        P.d_W = dalloc<float>(3 * (size_t)n); P.d_F = dalloc<float>(3 * (size_t)n);
        P.d_M = dalloc<float>(3 * (size_t)n);
        C.N = cn;
        C.d_IP = dalloc<uint32_t>(n); C.d_CI = dalloc<uint32_t>(n);
        C.d_CIs = dalloc<uint32_t>(2 * (size_t)n); C.d_pnC = dalloc<uint32_t>(2 * (size_t)cn);
        C.dtmpN_old = 128;
        CK(cudaMalloc(&C.d_tmp_old, C.dtmpN_old));
        A.bloks = n / SMEMDIM + 1;
        A.gencreated = 1;   // no cuRAND generator is needed here
        size_t nk = (size_t)n * k;
        IL.IonP = k; IL.N = (uint32_t)nk;
        IL.d_IL = dalloc<uint32_t>(nk, 0xFF);
        IL.d_ILtype = dalloc<uint8_t>(nk);
        IL.d_1d_iL = dalloc<float>(nk);
        IL.d_rij = dalloc<float3>(nk); IL.d_Oijt = dalloc<float3>(nk); IL.d_Fijn = dalloc<float3>(nk);
        IL.d_Fijt = dalloc<float3>(nk); IL.d_Mijn = dalloc<float3>(nk); IL.d_Mijt = dalloc<float3>(nk);
        IL.d_Mijadd = dalloc<float3>(nk);
        // d_FillIndex (md_calculate_cell.cu:13-26), as cbc_createCD launches it
        d_FillIndex<<<A.bloks, SMEMDIM>>>(C.d_IP, n);
        CK(cudaGetLastError());
        return 0;
    }
    void release() {
        void* ps[] = {P.d_R, P.d_V, P.d_W, P.d_F, P.d_M, C.d_IP, C.d_CI, C.d_CIs, C.d_pnC, C.d_tmp_old,
                      IL.d_IL, IL.d_ILtype, IL.d_1d_iL, IL.d_rij, IL.d_Oijt, IL.d_Fijn, IL.d_Fijt,
                      IL.d_Mijn, IL.d_Mijt, IL.d_Mijadd};
        for (void* p : ps) if (p) cudaFree(p);
    }
    size_t nk() const { return (size_t)N * K; }
};
}  // namespace

extern "C" {

// CellDistribution (md_cell_distribution.cu:52-101) on host positions.
int ref_cell_distribution(const float* hR, uint32_t N, uint32_t* hCI, uint32_t* hCIs, uint32_t* hpnC,
                          uint32_t CN, float a, float inv_a, rf_uint3 cN) {
    Dev d;
    if (d.alloc(N, 1, CN)) return -1;
    d.C.a = a; d.C._1d_a = inv_a; d.C.Nr = make_uint3(cN.x, cN.y, cN.z);
    if (up(d.P.d_R, hR, 3 * (size_t)N)) return -1;
    CellDistribution(d.P, d.A, d.S, d.C);
    CK(cudaDeviceSynchronize());
    int rc = down(hCI, d.C.d_CI, N) | down(hCIs, d.C.d_CIs, 2 * (size_t)N) | down(hpnC, d.C.d_pnC, 2 * (size_t)CN);
    d.release();
    return rc;
}

// InteractionListConstruct (md_interaction_list_construction.cu:163-168) after CellDistribution.
int ref_list_construct(const float* hR, uint32_t N, uint32_t K, uint32_t CN, float a, float inv_a, float aacut,
                       rf_uint3 cN, uint32_t* hIL) {
    Dev d;
    if (d.alloc(N, K, CN)) return -1;
    d.C.a = a; d.C._1d_a = inv_a; d.C.Nr = make_uint3(cN.x, cN.y, cN.z);
    d.IL.aacut = aacut;
    if (up(d.P.d_R, hR, 3 * (size_t)N)) return -1;
    CellDistribution(d.P, d.A, d.S, d.C);
    InteractionListConstruct(d.P, d.A, d.S, d.IL, d.C);
    CK(cudaDeviceSynchronize());
    int rc = down(hIL, d.IL.d_IL, d.nk());
    d.release();
    return rc;
}

// CellDistribution + InteractionListReConstructBPM (md_interaction_list_construction.cu:176-180)
// on a given row state.
int ref_reconstruct_bpm(const float* hR, uint32_t N, uint32_t K, uint32_t CN, float a, float inv_a, float aacut,
                        rf_uint3 cN, uint32_t* hIL, uint8_t* hType) {
    Dev d;
    if (d.alloc(N, K, CN)) return -1;
    d.C.a = a; d.C._1d_a = inv_a; d.C.Nr = make_uint3(cN.x, cN.y, cN.z);
    d.IL.aacut = aacut;
    if (up(d.P.d_R, hR, 3 * (size_t)N) || up(d.IL.d_IL, hIL, d.nk()) || up(d.IL.d_ILtype, hType, d.nk())) return -1;
    CellDistribution(d.P, d.A, d.S, d.C);
    InteractionListReConstructBPM(d.P, d.A, d.S, d.IL, d.C);
    CK(cudaDeviceSynchronize());
    int rc = down(hIL, d.IL.d_IL, d.nk()) | down(hType, d.IL.d_ILtype, d.nk());
    d.release();
    return rc;
}

// d_ConstructBoundInteractions (md_boundinteractions_construct.cu:35-106), launch as the drivers do.
int ref_construct_bonds(const float* hR, uint32_t N, uint32_t K, const uint32_t* hIL, uint8_t* hType, float* hiL,
                        float aa_create, float b_r) {
    Dev d;
    if (d.alloc(N, K, 1)) return -1;
    if (up(d.P.d_R, hR, 3 * (size_t)N) || up(d.IL.d_IL, hIL, d.nk()) || up(d.IL.d_ILtype, hType, d.nk()) ||
        up(d.IL.d_1d_iL, hiL, d.nk())) return -1;
    d_ConstructBoundInteractions<<<d.A.bloks, SMEMDIM>>>(d.P.d_R, d.P.d_V, d.P.d_W, d.IL.d_IL, d.IL.d_ILtype,
        d.IL.d_1d_iL, d.IL.d_rij, d.IL.d_Oijt, d.IL.d_Fijn, d.IL.d_Fijt, d.IL.d_Mijn, d.IL.d_Mijt, d.IL.d_Mijadd,
        N, K, aa_create, b_r);
    CK(cudaDeviceSynchronize());
    int rc = down(hType, d.IL.d_ILtype, d.nk()) | down(hiL, d.IL.d_1d_iL, d.nk());
    d.release();
    return rc;
}

// d_CalculateForcesDEM_22 then d_CalculateForcesDEM_21 on zeroed F, M, launched as the
// drivers launch them (md_calculationbraziltest.cu:172-177). which: 1 = _22 only,
// 2 = _21 only, 3 = both.
int ref_forces(const float* hR, const float* hV, const float* hW, uint32_t N, uint32_t K, const uint32_t* hIL,
               uint8_t* hType, const float* hiL, float* hRij, float* hOijt, float* hMijn, float* hMijt,
               float* hF, float* hM, const float* p22 /* dt,m_E,m_G,b_r,Gcn,Gct */,
               const float* p21 /* dt,hm_E,hm_G,p_A,mu,mur,mP,rP */, int which) {
    Dev d;
    if (d.alloc(N, K, 1)) return -1;
    size_t nk = d.nk();
    if (up(d.P.d_R, hR, 3 * (size_t)N) || up(d.P.d_V, hV, 3 * (size_t)N) || up(d.P.d_W, hW, 3 * (size_t)N) ||
        up(d.IL.d_IL, hIL, nk) || up(d.IL.d_ILtype, hType, nk) || up(d.IL.d_1d_iL, hiL, nk) ||
        up(d.IL.d_rij, (const float3*)hRij, nk) || up(d.IL.d_Oijt, (const float3*)hOijt, nk) ||
        up(d.IL.d_Mijn, (const float3*)hMijn, nk) || up(d.IL.d_Mijt, (const float3*)hMijt, nk)) return -1;
    if (which & 1)
        d_CalculateForcesDEM_22<<<4 * d.A.bloks, 256>>>(d.P.d_R, d.P.d_V, d.P.d_W, d.IL.d_IL, d.IL.d_ILtype,
            d.IL.d_1d_iL, d.IL.d_rij, d.IL.d_Oijt, d.IL.d_Mijn, d.IL.d_Mijt, d.P.d_F, d.P.d_M, N, K,
            p22[0], p22[1], p22[2], p22[3], p22[4], p22[5]);
    if (which & 2)
        d_CalculateForcesDEM_21<<<d.A.bloks, SMEMDIM>>>(d.P.d_R, d.P.d_V, d.P.d_W, d.IL.d_IL, d.IL.d_ILtype,
            d.IL.d_1d_iL, d.IL.d_rij, d.IL.d_Oijt, d.P.d_F, d.P.d_M, N, K,
            p21[0], p21[1], p21[2], p21[3], p21[4], p21[5], p21[6], p21[7]);
    CK(cudaDeviceSynchronize());
    int rc = down(hType, d.IL.d_ILtype, nk) | down((float3*)hRij, d.IL.d_rij, nk) |
             down((float3*)hOijt, d.IL.d_Oijt, nk) | down((float3*)hMijn, d.IL.d_Mijn, nk) |
             down((float3*)hMijt, d.IL.d_Mijt, nk) | down(hF, d.P.d_F, 3 * (size_t)N) | down(hM, d.P.d_M, 3 * (size_t)N);
    d.release();
    return rc;
}

// A whole test, in the order of the driver loop (md_calculationbraziltest.cu:132-198,
// md_calculationuniaxialcompression.cu:132-190), using the reference's kernels, its
// host step functions and its compression_data methods. t must be prepared.
// Returns steps taken (>= 0) or -1.
long long ref_run(rf_task* t, const float* hR0, uint32_t max_steps, float* hR, float* hV, float* hW,
                  uint32_t* hIL, uint8_t* hType, float* hiL, float* hRij, float* hOijt, float* hMijn,
                  float* hMijt, double* curve, uint64_t cap, uint64_t* nsaved) {
    md_task_data m;
    std::memset(&m.Po, 0, sizeof(m.Po));
    potential_data& Po = m.Po;
    const rf_potential& P = t->Po;
    Po.m_E = P.m_E; Po.m_nu = P.m_nu; Po.m_Ec = P.m_Ec; Po.m_Gc = P.m_Gc; Po.m_ro = P.m_ro; Po.b_r = P.b_r;
    Po.b_d = P.b_d; Po.p_r = P.p_r; Po.p_e = P.p_e; Po.p_mu = P.p_mu; Po.p_mur = P.p_mur; Po.a_farcut = P.a_farcut;
    Po.CalculateParameters();
    // sample_data as the caller left it (copied from the prepared task)
    sample_data& S = m.S;
    const rf_sample& s = t->S;
#define F3(dst, src) dst = make_float3(src.x, src.y, src.z)
#define D3(dst, src) dst = make_double3(src.x, src.y, src.z)
    D3(S.A_real, s.A_real); D3(S.B_real, s.B_real); D3(S.size_real, s.size_real); D3(S.center_real, s.center_real);
    S.Vext = s.Vext;
    F3(S.L, s.L); F3(S.A, s.A); F3(S.B, s.B); F3(S.axis, s.axis); F3(S.center, s.center); F3(S.size, s.size);
    F3(S.sized2, s.sized2); F3(S.hidenpoint, s.hidenpoint); F3(S.spacesize, s.spacesize);
    F3(S.spacesized2, s.spacesized2);
    S.R0 = s.R0; S.H0 = s.H0; S.Vgenmax = s.Vgenmax;
    m.C.a = t->C.a;
    m.P.N = (uint32_t)t->N;
    m.IL.IonP = t->K;
    bool brazil = (t->kind == RF_TEST_BRAZIL);
    m.Compress.VLoad = t->Compress.VLoad;
    if (brazil) m.Compress.CalculateBParameters(S.size_real, S.center_real, Po, t->Compress.MinStress, t->Compress.MaxStrain);
    else m.Compress.CalculateUParameters(S.size_real, S.center_real, Po, t->Compress.MinStress, t->Compress.MaxStrain);
    m.Compress.V = 0.0;        // read before the first CompressU/B sets it
    m.Compress.Strain = 0.0;
    // h_Calculation*: parameters (:117-120)
    m.IL.CalculateParameters(m.P.N, Po.a_farcut);
    m.C.CalculateParameters(m.S.B.x, m.S.B.y, m.S.B.z);
    Dev d;
    if (d.alloc(m.P.N, m.IL.IonP, m.C.N)) return -1;
    d.C.a = m.C.a; d.C._1d_a = m.C._1d_a; d.C.Nr = m.C.Nr; d.C.N = m.C.N;
    d.IL.acut = m.IL.acut; d.IL.aacut = m.IL.aacut;
    uint32_t N = m.P.N, K = m.IL.IonP;
    additional_data& A = d.A;
    result_data R{};
    R.Nsave = 1000000; R.dNsave = 1;
    ResultsUInit(d.P, A, S, d.C, R, m.Compress);
    if (up(d.P.d_R, hR0, 3 * (size_t)N)) return -1;
    CellDistribution(d.P, A, S, d.C);
    InteractionListConstruct(d.P, A, S, d.IL, d.C);
    d_ConstructBoundInteractions<<<A.bloks, SMEMDIM>>>(d.P.d_R, d.P.d_V, d.P.d_W, d.IL.d_IL, d.IL.d_ILtype,
        d.IL.d_1d_iL, d.IL.d_rij, d.IL.d_Oijt, d.IL.d_Fijn, d.IL.d_Fijt, d.IL.d_Mijn, d.IL.d_Mijt, d.IL.d_Mijadd,
        N, K, Po.b_dd, Po.b_r);
    d_DeleteFarLinks<<<A.bloks, SMEMDIM>>>(d.P.d_R, N, d.IL.d_IL, d.IL.d_ILtype, d.IL.d_1d_iL, d.IL.d_rij,
        d.IL.d_Oijt, d.IL.d_Fijn, d.IL.d_Fijt, d.IL.d_Mijn, d.IL.d_Mijt, d.IL.d_Mijadd, K, Po.aa_farcut);
    R.stepsave = 0;
    uint32_t steps;
    compression_data& Cp = m.Compress;
    for (steps = 0; Cp.Strain < Cp.MaxStrain && !Cp.Fracture && (max_steps == 0 || steps < max_steps); ++steps) {
        CellDistribution(d.P, A, S, d.C);
        InteractionListReConstructBPM(d.P, A, S, d.IL, d.C);
        cudaMemset(d.P.d_F, 0, 3 * (size_t)N * sizeof(float));
        cudaMemset(d.P.d_M, 0, 3 * (size_t)N * sizeof(float));
        d_CalculateForcesDEM_22<<<4 * A.bloks, 256>>>(d.P.d_R, d.P.d_V, d.P.d_W, d.IL.d_IL, d.IL.d_ILtype,
            d.IL.d_1d_iL, d.IL.d_rij, d.IL.d_Oijt, d.IL.d_Mijn, d.IL.d_Mijt, d.P.d_F, d.P.d_M, N, K, Po.dt, Po.m_E,
            Po.m_G, Po.b_r, Po.m_Ec, Po.m_Gc);
        d_CalculateForcesDEM_21<<<A.bloks, SMEMDIM>>>(d.P.d_R, d.P.d_V, d.P.d_W, d.IL.d_IL, d.IL.d_ILtype,
            d.IL.d_1d_iL, d.IL.d_rij, d.IL.d_Oijt, d.P.d_F, d.P.d_M, N, K, Po.dt, Po.hm_E, Po.hm_G, Po.p_A,
            Po.p_mu, Po.p_mur, Po.p_m, Po.p_r);
        if (brazil)
            d_braziltest_simple2<<<A.bloks, SMEMDIM>>>(d.P.d_R, d.P.d_V, d.P.d_F, R.d_FL, N, Cp.center, Cp.RR,
                Cp.Top, Cp.Bottom, Cp.TopR, Cp.BottomR, Cp.V, S.center.y + S.spacesized2.y);
        else
            d_UniaxialCompression3_simple<<<A.bloks, SMEMDIM>>>(d.P.d_R, d.P.d_V, d.P.d_F, R.d_FL, N, Cp.center,
                Cp.RR, Cp.Top, Cp.Bottom, Cp.TopR, Cp.BottomR, Cp.V, S.center.z + S.spacesized2.z);
        SumForcesULoading(R, Cp, steps);
        d_CalculateIncrementsDEM<<<A.bloks, SMEMDIM>>>(d.P.d_F, d.P.d_V, d.P.d_R, d.P.d_M, d.P.d_W, N, Po.dt_d_m,
            Po.dt, Po.dt_d_I);
        d_ParallelepipedCutRestriction<<<A.bloks, SMEMDIM>>>(d.P.d_R, d.P.d_V, d.P.d_F, N, S.center,
            S.spacesized2, S.hidenpoint);
        d_DeleteFarLinks<<<A.bloks, SMEMDIM>>>(d.P.d_R, N, d.IL.d_IL, d.IL.d_ILtype, d.IL.d_1d_iL, d.IL.d_rij,
            d.IL.d_Oijt, d.IL.d_Fijn, d.IL.d_Fijt, d.IL.d_Mijn, d.IL.d_Mijt, d.IL.d_Mijadd, K, Po.aa_farcut);
        if (brazil) Cp.CompressB(Cp.Stress, Po);
        else Cp.CompressU(Cp.Stress, Po);
    }
    CK(cudaDeviceSynchronize());
    size_t nk = (size_t)N * K;
    int rc = down(hR, d.P.d_R, 3 * (size_t)N) | down(hV, d.P.d_V, 3 * (size_t)N) | down(hW, d.P.d_W, 3 * (size_t)N) |
             down(hIL, d.IL.d_IL, nk) | down(hType, d.IL.d_ILtype, nk) | down(hiL, d.IL.d_1d_iL, nk) |
             down((float3*)hRij, d.IL.d_rij, nk) | down((float3*)hOijt, d.IL.d_Oijt, nk) |
             down((float3*)hMijn, d.IL.d_Mijn, nk) | down((float3*)hMijt, d.IL.d_Mijt, nk);
    if (curve) {
        uint64_t n = R.stepsave < cap ? R.stepsave : cap;
        std::memcpy(curve, R.h_sFL, 3 * n * sizeof(double));
    }
    if (nsaved) *nsaved = R.stepsave;
    t->Compress.FractureStress = Cp.FractureStress;
    t->Compress.FractureStrain = Cp.FractureStrain;
    t->Compress.Fracture = Cp.Fracture;
    t->Compress.Stress = Cp.Stress;
    t->Compress.Strain = Cp.Strain;
    t->Compress.Loading = Cp.Loading;
    ResultsUDelete(R);
    d.release();
    return rc ? -1 : (long long)steps;
}

}  // extern "C"
