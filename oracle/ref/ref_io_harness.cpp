// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// Calls the reference's own writers, compiled unmodified from its sources into
// oracle/_ref/libmdref_io.so: SaveLammpsDATASimple (md_savelammpsdata.cpp:8-74) and
// SaveAllData (md_savealldata.cpp:12-36, which writes ./result/DATA.dat relative to the
// working directory). The tests compare their files with the engine library's writers
// byte for byte. SaveAllData first copies the device arrays to the host ones with
// cudaMemcpy; the harness gives it no device arrays (null pointers), so those copies
// fail, the reference's HANDLE_ERROR reports and continues, and the host arrays the
// harness filled are what it writes. The tests call it only where no GPU is visible.

#include <cstring>
#include <unistd.h>
#include "md.h"

extern "C" {

int ref_save_lammps(const char* path, uint32_t N, uint32_t K, const float* R, const float* V, const float* W,
                    const uint32_t* IL, const uint8_t* ILtype, const float A[3], const float B[3], double dt,
                    double p_m, double p_I, int flagv) {
    particle_data P;
    std::memset(&P, 0, sizeof(P));
    P.h_R = const_cast<float*>(R); P.h_V = const_cast<float*>(V); P.h_W = const_cast<float*>(W);
    P.N = N;
    cell_data Cd;
    std::memset(&Cd, 0, sizeof(Cd));
    sample_data S;
    std::memset(&S, 0, sizeof(S));
    S.A = make_float3(A[0], A[1], A[2]);
    S.B = make_float3(B[0], B[1], B[2]);
    additional_data Ad;
    interaction_list_data ILd;
    std::memset(&ILd, 0, sizeof(ILd));
    ILd.h_IL = const_cast<uint32_t*>(IL);
    ILd.h_ILtype = const_cast<uint8_t*>(ILtype);
    ILd.IonP = K;
    ILd.N = N * K;
    potential_data Po;
    std::memset(&Po, 0, sizeof(Po));
    Po.dt = dt; Po.p_m = p_m; Po.p_I = p_I;
    char name[1024];
    std::strncpy(name, path, sizeof(name) - 1);
    name[sizeof(name) - 1] = 0;
    SaveLammpsDATASimple(P, Cd, S, Ad, ILd, Po, name, flagv != 0);
    return 0;
}

// sample: L, A, B, axis, center, size as 18 floats, then R0, H0, Vgenmax; pn: S.PN
int ref_save_all(const char* dir, const float* sample, uint32_t pn, uint32_t N, uint32_t K, float acut,
                 const float* F, const float* V, const float* R, const float* M, const float* W, const float* Q,
                 const uint32_t* IL, const uint8_t* ILtype, const float* iL, const float* slots /* 7 x 3NK */) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd)) || chdir(dir) != 0) return -1;
    sample_data S;
    std::memset(&S, 0, sizeof(S));
    float3* v3[6] = {&S.L, &S.A, &S.B, &S.axis, &S.center, &S.size};
    for (int q = 0; q < 6; ++q) *v3[q] = make_float3(sample[3 * q], sample[3 * q + 1], sample[3 * q + 2]);
    S.R0 = sample[18]; S.H0 = sample[19]; S.Vgenmax = sample[20];
    S.PN = pn;
    particle_data P;
    std::memset(&P, 0, sizeof(P));
    P.N = N;
    P.h_F = const_cast<float*>(F); P.h_V = const_cast<float*>(V); P.h_R = const_cast<float*>(R);
    P.h_M = const_cast<float*>(M); P.h_W = const_cast<float*>(W);
    P.h_Q = reinterpret_cast<float4*>(const_cast<float*>(Q));
    interaction_list_data ILd;
    std::memset(&ILd, 0, sizeof(ILd));
    const size_t NK = (size_t)N * K;
    ILd.N = (uint32_t)NK; ILd.IonP = K; ILd.acut = acut;
    ILd.h_IL = const_cast<uint32_t*>(IL);
    ILd.h_ILtype = const_cast<uint8_t*>(ILtype);
    ILd.h_1d_iL = const_cast<float*>(iL);
    float3* s3 = reinterpret_cast<float3*>(const_cast<float*>(slots));
    ILd.h_rij = s3; ILd.h_Oijt = s3 + NK; ILd.h_Fijn = s3 + 2 * NK; ILd.h_Fijt = s3 + 3 * NK;
    ILd.h_Mijn = s3 + 4 * NK; ILd.h_Mijt = s3 + 5 * NK; ILd.h_Mijadd = s3 + 6 * NK;
    cell_data Cd;
    std::memset(&Cd, 0, sizeof(Cd));
    additional_data Ad;
    potential_data Po;
    std::memset(&Po, 0, sizeof(Po));
    SaveAllData(P, Cd, S, Ad, ILd, Po);
    return chdir(cwd) == 0 ? 0 : -1;
}

}  // extern "C"
