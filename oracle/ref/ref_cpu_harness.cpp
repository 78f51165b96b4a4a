// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// Timing harness around the reference's own CPU bond-force path,
// h_CalculateForceElastic (md_calculateforcesbpm_cpu.cpp:20-288), compiled from
// the reference source unmodified into oracle/_ref/libmdref_cpu.so. It implements
// an older, sign-flipped bond model (it is not the live GPU formula), so it serves
// as the timed CPU baseline only, never as a parity oracle.
//
// The function compares every result against per-slot arrays the live GPU path no
// longer fills and prints a line for each mismatch; std::cerr has its buffer
// detached for the call, so those prints return at once (no formatting, no flush,
// no stderr lock). The slot arrays are only read by the function (its writes are
// commented out in the source), so the threads share them; each thread owns F, M.

#include <chrono>
#include <cstring>
#include <iostream>
#include <thread>
#include <vector>
#include "md.h"

extern "C" {

// Runs h_CalculateForceElastic `reps` times over the bond slots of one specimen on
// `threads` host threads, each thread on its own copy of the mutable state (the
// function walks all N*K slots of one specimen and cannot be split). Returns the
// wall time in seconds; *slot_evals gets the bond-slot evaluations done.
static double run_bond_forces(const float* R, const float* V, const float* W, const uint32_t* IL,
                              const uint8_t* ILtype, const float* iL, uint32_t N, uint32_t K, float dt,
                              float m_E, float m_G, const float* slot_b_r, float b_r, float m_Gcritn,
                              float m_Gcritt, int reps, int threads, uint64_t* slot_evals);

double ref_cpu_bond_forces(const float* R, const float* V, const float* W, const uint32_t* IL,
                           const uint8_t* ILtype, const float* iL, uint32_t N, uint32_t K, float dt,
                           float m_E, float m_G, float b_r, float m_Gcritn, float m_Gcritt, int reps,
                           int threads, uint64_t* slot_evals) {
    return run_bond_forces(R, V, W, IL, ILtype, iL, N, K, dt, m_E, m_G, nullptr, b_r, m_Gcritn, m_Gcritt, reps,
                           threads, slot_evals);
}

// The same with a bond radius per slot (slot_b_r[N*K]), as the function's per-slot ab_r
// and AxialMoment arguments allow: a polydisperse specimen's bonds each have their own.
double ref_cpu_bond_forces_rb(const float* R, const float* V, const float* W, const uint32_t* IL,
                              const uint8_t* ILtype, const float* iL, uint32_t N, uint32_t K, float dt,
                              float m_E, float m_G, const float* slot_b_r, float m_Gcritn, float m_Gcritt, int reps,
                              int threads, uint64_t* slot_evals) {
    return run_bond_forces(R, V, W, IL, ILtype, iL, N, K, dt, m_E, m_G, slot_b_r, 0.f, m_Gcritn, m_Gcritt, reps,
                           threads, slot_evals);
}

}  // extern "C"

static double run_bond_forces(const float* R, const float* V, const float* W, const uint32_t* IL,
                              const uint8_t* ILtype, const float* iL, uint32_t N, uint32_t K, float dt,
                              float m_E, float m_G, const float* slot_b_r, float b_r, float m_Gcritn,
                              float m_Gcritt, int reps, int threads, uint64_t* slot_evals) {
    const size_t nk = (size_t)N * K;
    uint64_t bonds = 0;
    for (size_t k = 0; k < nk; ++k) if (IL[k] < N && ILtype[k] == 1) ++bonds;
    const float PI = 3.14159265358979f;
    std::vector<float> ab_r(nk, b_r), axial(nk, PI * b_r * b_r * b_r * b_r * 0.25f);
    if (slot_b_r)
        for (size_t k = 0; k < nk; ++k) {
            const float r = slot_b_r[k];
            ab_r[k] = r;
            axial[k] = PI * r * r * r * r * 0.25f;
        }
    if (threads < 1) threads = 1;
    float3 z = make_float3(0.f, 0.f, 0.f);
    std::vector<float3> Rij(nk, z), Oijt(nk, z), Mijn(nk, z), Mijt(nk, z), Fij(nk, z), Fijn(nk, z), Fijt(nk, z),
        Mijadd(nk, z);
    interaction_list_data ILd;
    particle_data Pd;
    std::memset(&ILd, 0, sizeof(ILd));
    std::memset(&Pd, 0, sizeof(Pd));
    ILd.h_IL = const_cast<uint32_t*>(IL);
    ILd.h_ILtype = const_cast<uint8_t*>(ILtype);
    ILd.h_Fijn = Fijn.data(); ILd.h_Fijt = Fijt.data(); ILd.h_Mijn = Mijn.data();
    ILd.h_Mijt = Mijt.data(); ILd.h_Mijadd = Mijadd.data();
    ILd.IonP = K; ILd.N = (uint32_t)nk;
    Pd.N = N;
    std::vector<std::vector<float>> F(threads, std::vector<float>(3 * (size_t)N, 0.f)),
        M(threads, std::vector<float>(3 * (size_t)N, 0.f));
    std::streambuf* saved = std::cerr.rdbuf(nullptr);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t]() {
            for (int r = 0; r < reps; ++r)
                h_CalculateForceElastic(R, V, W, F[t].data(), M[t].data(), ab_r.data(), iL, axial.data(),
                                        Rij.data(), Oijt.data(), Mijn.data(), Mijt.data(), Fij.data(),
                                        N, ILd, Pd, dt, m_E, m_G, m_Gcritn, m_Gcritt);
        });
    for (auto& th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    std::cerr.rdbuf(saved);
    std::cerr.clear();
    if (slot_evals) *slot_evals = bonds * (uint64_t)reps * (uint64_t)threads;
    return std::chrono::duration<double>(t1 - t0).count();
}
