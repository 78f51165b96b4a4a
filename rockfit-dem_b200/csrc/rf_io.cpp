// Specimen state files: the reference's binary state dump and its LAMMPS data export.
//
// rf_save_all_data / rf_load_all_data write and read the byte layout of the reference's
// SaveAllData / LoadAllData (md_savealldata.cpp:12-91 with write_sample_data :98-111,
// write_particle_data :127-142, write_interaction_list_data :176-199 and their readers),
// so a state saved here loads in the reference and the other way round. Ids and counts
// are written with the width of the build that made the file: 4 bytes for the reference's
// own (MSVC) build, 8 for a Linux build of it.
//
// rf_save_lammps_data writes the text of SaveLammpsDATASimple (md_savelammpsdata.cpp:8-74):
// header, box, atoms in metres, per-atom translational and rotational energies (joules),
// and every directed bond slot.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <istream>
#include <ostream>
#include <vector>

#include "../../include/rockfit_b200.h"

namespace rf {
void set_error(const char* fmt, ...);
}
using rf::set_error;

namespace {

constexpr double kLength = 1e-3;        // mm -> m (md_phys_constants.h length_const)
constexpr double kEnergy = 1.0;         // force_const (1e3) * length_const (1e-3): mg mm^2/us^2 -> J

void put_id(std::ostream& f, uint64_t v, int id_bytes) {
    if (id_bytes == 4) {
        const uint32_t w = (uint32_t)v;
        f.write((const char*)&w, 4);
    } else {
        f.write((const char*)&v, 8);
    }
}

bool get_id(std::istream& f, uint64_t* v, int id_bytes) {
    if (id_bytes == 4) {
        uint32_t w = 0;
        f.read((char*)&w, 4);
        *v = w;
    } else {
        f.read((char*)v, 8);
    }
    return (bool)f;
}

template <class T>
void put(std::ostream& f, const T* p, size_t n, std::vector<char>& zeros) {
    const size_t bytes = n * sizeof(T);
    if (p) {
        f.write((const char*)p, (std::streamsize)bytes);
    } else {
        if (zeros.size() < bytes) zeros.assign(bytes, 0);
        f.write(zeros.data(), (std::streamsize)bytes);
    }
}

template <class T>
bool get(std::istream& f, T* p, size_t n) {
    if (p) {
        f.read((char*)p, (std::streamsize)(n * sizeof(T)));
    } else {
        f.seekg((std::streamoff)(n * sizeof(T)), std::ios::cur);
    }
    return (bool)f;
}

}  // namespace

namespace rf {

// The SaveAllData payload on an open stream (rf_save_all_data; a checkpoint's body).
rf_status io_write_all(std::ostream& f, int id_bytes, const rf_sample* S, uint64_t pn, uint64_t N, uint32_t K,
                       float acut, const float* F, const float* V, const float* R, const float* M, const float* W,
                       const float* Q, const uint_fast32_t* IL, const uint8_t* ILtype, const float* _1d_iL,
                       const rf_float3* Rij, const rf_float3* Oijt, const rf_float3* Fijn, const rf_float3* Fijt,
                       const rf_float3* Mijn, const rf_float3* Mijt, const rf_float3* Mijadd) {
    if (!S || (id_bytes != 4 && id_bytes != 8) || N == 0 || K == 0 || !R || !IL || !ILtype) {
        set_error("rf_save_all_data: bad arguments");
        return RF_ERR_INVALID;
    }
    std::vector<char> zeros;
    // write_sample_data: six float3, then R0 and H0 each written as a float3 -- the 12
    // bytes from R0 (R0, H0, Vgenmax) and the 12 from H0 (H0, Vgenmax and the 4 bytes
    // after Vgenmax: PN with 4-byte ids, alignment padding (written as 0) with 8-byte ids)
    const rf_float3* v3[6] = {&S->L, &S->A, &S->B, &S->axis, &S->center, &S->size};
    for (const rf_float3* p : v3) f.write((const char*)p, sizeof(rf_float3));
    const uint32_t tail = id_bytes == 4 ? (uint32_t)pn : 0u;
    float r0[3] = {S->R0, S->H0, S->Vgenmax};
    float h0[3] = {S->H0, S->Vgenmax, 0.f};
    std::memcpy(&h0[2], &tail, 4);
    f.write((const char*)r0, sizeof(r0));
    f.write((const char*)h0, sizeof(h0));
    // write_particle_data
    put_id(f, N, id_bytes);
    const size_t n3 = 3 * (size_t)N;
    put(f, F, n3, zeros); put(f, V, n3, zeros); put(f, R, n3, zeros); put(f, M, n3, zeros); put(f, W, n3, zeros);
    put(f, Q, 4 * (size_t)N, zeros);
    // write_interaction_list_data
    const size_t NK = (size_t)N * K;
    put_id(f, NK, id_bytes);
    put_id(f, K, id_bytes);
    f.write((const char*)&acut, sizeof(float));
    if (id_bytes == (int)sizeof(uint_fast32_t)) {
        f.write((const char*)IL, (std::streamsize)(NK * sizeof(uint_fast32_t)));
    } else {
        std::vector<char> buf(NK * (size_t)id_bytes);
        for (size_t k = 0; k < NK; ++k) {
            const uint64_t v = (uint64_t)IL[k];
            if (id_bytes == 4) { const uint32_t w = (uint32_t)v; std::memcpy(&buf[4 * k], &w, 4); }
            else std::memcpy(&buf[8 * k], &v, 8);
        }
        f.write(buf.data(), (std::streamsize)buf.size());
    }
    f.write((const char*)ILtype, (std::streamsize)NK);
    put(f, _1d_iL, NK, zeros);
    const rf_float3* slots[7] = {Rij, Oijt, Fijn, Fijt, Mijn, Mijt, Mijadd};
    for (const rf_float3* p : slots) put(f, p, NK, zeros);
    if (!f) { set_error("rf_save_all_data: write failed"); return RF_ERR_INVALID; }
    return RF_OK;
}

// The SaveAllData payload from an open stream (rf_load_all_data; a checkpoint's body).
rf_status io_read_all(std::istream& f, int id_bytes, rf_sample* S, uint64_t* pn, uint64_t* N_out, uint32_t* K_out,
                      float* acut, float* F, float* V, float* R, float* M, float* W, float* Q, uint_fast32_t* IL,
                      uint8_t* ILtype, float* _1d_iL, rf_float3* Rij, rf_float3* Oijt, rf_float3* Fijn,
                      rf_float3* Fijt, rf_float3* Mijn, rf_float3* Mijt, rf_float3* Mijadd) {
    if ((id_bytes != 4 && id_bytes != 8) || !N_out || !K_out) {
        set_error("rf_load_all_data: bad arguments");
        return RF_ERR_INVALID;
    }
    rf_sample s;
    std::memset(&s, 0, sizeof(s));
    rf_float3* v3[6] = {&s.L, &s.A, &s.B, &s.axis, &s.center, &s.size};
    for (rf_float3* p : v3) f.read((char*)p, sizeof(rf_float3));
    float r0[3], h0[3];
    f.read((char*)r0, sizeof(r0));
    f.read((char*)h0, sizeof(h0));
    s.R0 = r0[0];
    s.H0 = h0[0];
    s.Vgenmax = h0[1];
    uint32_t tail = 0;
    std::memcpy(&tail, &h0[2], 4);
    uint64_t N = 0, NK = 0, K = 0;
    if (!get_id(f, &N, id_bytes) || N == 0) { set_error("rf_load_all_data: bad particle count"); return RF_ERR_INVALID; }
    // sizes only: the caller allocates, then calls again with buffers
    const bool sizes_only = !R;
    const size_t n3 = 3 * (size_t)N;
    if (sizes_only) {
        f.seekg((std::streamoff)(5 * n3 * sizeof(float) + 4 * (size_t)N * sizeof(float)), std::ios::cur);
    } else {
        get(f, F, n3); get(f, V, n3); get(f, R, n3); get(f, M, n3); get(f, W, n3); get(f, Q, 4 * (size_t)N);
    }
    if (!get_id(f, &NK, id_bytes) || !get_id(f, &K, id_bytes) || K == 0 || NK != N * K) {
        set_error("rf_load_all_data: bad interaction list header");
        return RF_ERR_INVALID;
    }
    float ac = 0.f;
    f.read((char*)&ac, sizeof(float));
    *N_out = N;
    *K_out = (uint32_t)K;
    if (acut) *acut = ac;
    if (pn) *pn = id_bytes == 4 ? tail : 0u;
    if (sizes_only) {
        if (!f) { set_error("rf_load_all_data: truncated file"); return RF_ERR_INVALID; }
        if (S) *S = s;
        return RF_OK;
    }
    if (!IL || !ILtype) { set_error("rf_load_all_data: IL and ILtype are required"); return RF_ERR_INVALID; }
    std::vector<char> buf(NK * (size_t)id_bytes);
    f.read(buf.data(), (std::streamsize)buf.size());
    for (size_t k = 0; k < NK; ++k) {
        uint64_t v = 0;
        if (id_bytes == 4) { uint32_t w; std::memcpy(&w, &buf[4 * k], 4); v = w == 0xFFFFFFFFu ? ~0ull : w; }
        else std::memcpy(&v, &buf[8 * k], 8);
        IL[k] = (uint_fast32_t)v;
    }
    get(f, ILtype, NK);
    get(f, _1d_iL, NK);
    rf_float3* slots[7] = {Rij, Oijt, Fijn, Fijt, Mijn, Mijt, Mijadd};
    for (rf_float3* p : slots) get(f, p, NK);
    if (!f) { set_error("rf_load_all_data: truncated file"); return RF_ERR_INVALID; }
    // LoadAllData (md_savealldata.cpp:62-85): the real extents from the loaded positions
    double lo[3] = {1e20, 1e20, 1e20}, hi[3] = {-1e20, -1e20, -1e20};
    for (uint64_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) {
            const double x = R[i + a * N];
            if (x < lo[a]) lo[a] = x;
            if (x > hi[a]) hi[a] = x;
        }
    s.A_real = rf_double3{lo[0], lo[1], lo[2]};
    s.B_real = rf_double3{hi[0], hi[1], hi[2]};
    s.size_real = rf_double3{hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    s.center_real = rf_double3{0.5 * (hi[0] + lo[0]), 0.5 * (hi[1] + lo[1]), 0.5 * (hi[2] + lo[2])};
    if (S) *S = s;
    return RF_OK;
}

}  // namespace rf

extern "C" {

rf_status rf_save_all_data(const char* path, int id_bytes, const rf_sample* S, uint64_t pn, uint64_t N, uint32_t K,
                           float acut, const float* F, const float* V, const float* R, const float* M,
                           const float* W, const float* Q, const uint_fast32_t* IL, const uint8_t* ILtype,
                           const float* _1d_iL, const rf_float3* Rij, const rf_float3* Oijt, const rf_float3* Fijn,
                           const rf_float3* Fijt, const rf_float3* Mijn, const rf_float3* Mijt,
                           const rf_float3* Mijadd) {
    if (!path) { set_error("rf_save_all_data: bad arguments"); return RF_ERR_INVALID; }
    std::ofstream f(path, std::ios::out | std::ios::binary | std::ios::trunc);
    if (!f) { set_error("rf_save_all_data: cannot open %s", path); return RF_ERR_INVALID; }
    const rf_status st = rf::io_write_all(f, id_bytes, S, pn, N, K, acut, F, V, R, M, W, Q, IL, ILtype, _1d_iL, Rij,
                                          Oijt, Fijn, Fijt, Mijn, Mijt, Mijadd);
    f.close();
    if (st == RF_OK && !f) { set_error("rf_save_all_data: write to %s failed", path); return RF_ERR_INVALID; }
    return st;
}

rf_status rf_load_all_data(const char* path, int id_bytes, rf_sample* S, uint64_t* pn, uint64_t* N_out,
                           uint32_t* K_out, float* acut, float* F, float* V, float* R, float* M, float* W, float* Q,
                           uint_fast32_t* IL, uint8_t* ILtype, float* _1d_iL, rf_float3* Rij, rf_float3* Oijt,
                           rf_float3* Fijn, rf_float3* Fijt, rf_float3* Mijn, rf_float3* Mijt, rf_float3* Mijadd) {
    if (!path) { set_error("rf_load_all_data: bad arguments"); return RF_ERR_INVALID; }
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) { set_error("rf_load_all_data: cannot open %s", path); return RF_ERR_INVALID; }
    return rf::io_read_all(f, id_bytes, S, pn, N_out, K_out, acut, F, V, R, M, W, Q, IL, ILtype, _1d_iL, Rij, Oijt,
                           Fijn, Fijt, Mijn, Mijt, Mijadd);
}

rf_status rf_save_lammps_data(const char* path, const rf_task* t, uint64_t N, uint32_t K, const float* R,
                              const float* V, const float* W, const uint_fast32_t* IL, const uint8_t* ILtype,
                              int with_energy) {
    if (!path || !t || N == 0 || K == 0 || !R || !IL || !ILtype || (with_energy && (!V || !W))) {
        set_error("rf_save_lammps_data: bad arguments");
        return RF_ERR_INVALID;
    }
    std::ofstream f(path, std::ios::out | std::ios::trunc);
    if (!f) { set_error("rf_save_lammps_data: cannot open %s", path); return RF_ERR_INVALID; }
    const size_t NK = (size_t)N * K;
    uint64_t nb = 0;
    for (size_t k = 0; k < NK; ++k) if ((uint64_t)IL[k] < N && ILtype[k] == 1) ++nb;
    const rf_sample& S = t->S;
    const rf_potential& P = t->Po;
    f << "LAMMPS Description T0=" << P.dt << "  (1st line of file)\n\n";
    f << N << " atoms\n" << nb << " bonds\n" << 0 << " angles\n" << 0 << " dihedrals\n" << 0 << " impropers\n";
    f << 1 << " atom types\n" << 2 << " bond types\n";
    f << S.A.x * kLength << " " << S.B.x * kLength << " xlo xhi\n" << S.A.y * kLength << " " << S.B.y * kLength
      << " ylo yhi\n" << S.A.z * kLength << " " << S.B.z * kLength << " zlo zhi\n";
    f << "Masses\n\n" << 1 << " " << 1.0 << "\n";
    f << "Bond Coeffs\n\n" << 2 << " " << 1.0 << " " << 2.0 << "\n\n";
    f << "Atoms\n\n";
    for (uint64_t i = 0; i < N; ++i)
        f << i + 1 << " " << "1 " << R[i] * kLength << " " << R[i + N] * kLength << " " << R[i + 2 * N] * kLength
          << "\n";
    f << "Velocities\n\n";
    for (uint64_t i = 0; i < N; ++i) {
        double Et = 0, Er = 0;
        if (with_energy) {
            const float v2 = V[i] * V[i] + V[i + N] * V[i + N] + V[i + 2 * N] * V[i + 2 * N];
            const float w2 = W[i] * W[i] + W[i + N] * W[i + N] + W[i + 2 * N] * W[i + 2 * N];
            Et = 0.5 * P.p_m * v2 * kEnergy;
            Er = 0.5 * P.p_I * w2 * kEnergy;
        }
        f << i + 1 << " " << Et << " " << Er << " " << Et + Er << "\n";
    }
    f << "\nBonds\n\n";
    uint64_t k = 1;
    for (size_t q = 0; q < NK; ++q) {
        if ((uint64_t)IL[q] < N && ILtype[q] == 1) {
            f << k << " " << ILtype[q] + 1 << " " << q / K + 1 << " " << (uint64_t)IL[q] + 1 << "\n";
            ++k;
        }
    }
    f.close();
    if (!f) { set_error("rf_save_lammps_data: write to %s failed", path); return RF_ERR_INVALID; }
    return RF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Particle positions as text (md_createcylindersample.cu:104-133, SaveParticleDATAtxt /
// LoadParticleDATAtxt): the count on the first line, then one line "x y z" per particle
// in metres -- each float coordinate (mm) times the length unit 1e-3 as a double, in the
// stream's default format (6 significant digits). Reading multiplies by 1 / 1e-3 and
// stores floats, planar x | y | z.
// ---------------------------------------------------------------------------
extern "C" rf_status rf_save_positions_txt(const char* path, const float* R, uint64_t n) {
    if (!path || (!R && n)) { rf::set_error("rf_save_positions_txt: bad arguments"); return RF_ERR_INVALID; }
    std::ofstream f(path, std::ios::out);
    if (!f) { rf::set_error("rf_save_positions_txt: cannot open %s", path); return RF_ERR_INVALID; }
    const double lc = 1e-3;
    f << n << "\n";
    for (uint64_t i = 0; i < n; ++i)
        f << R[i] * lc << " " << R[i + n] * lc << " " << R[i + 2 * n] * lc << "\n";
    f.close();
    if (!f) { rf::set_error("rf_save_positions_txt: write to %s failed", path); return RF_ERR_INVALID; }
    return RF_OK;
}

extern "C" rf_status rf_load_positions_txt(const char* path, float* R, uint64_t cap, uint64_t* n) {
    if (!path || !n) { rf::set_error("rf_load_positions_txt: bad arguments"); return RF_ERR_INVALID; }
    std::ifstream f(path, std::ios::in);
    if (!f) { rf::set_error("rf_load_positions_txt: cannot open %s", path); return RF_ERR_INVALID; }
    uint64_t m = 0;
    if (!(f >> m)) { rf::set_error("rf_load_positions_txt: %s has no particle count", path); return RF_ERR_INVALID; }
    *n = m;
    if (!R) return RF_OK;
    if (cap < m) { rf::set_error("rf_load_positions_txt: capacity %llu < %llu particles", (unsigned long long)cap, (unsigned long long)m); return RF_ERR_CAPACITY; }
    const double lc = 1.0 / 1e-3;
    for (uint64_t i = 0; i < m; ++i) {
        double x, y, z;
        if (!(f >> x >> y >> z)) { rf::set_error("rf_load_positions_txt: %s ends at particle %llu", path, (unsigned long long)i); return RF_ERR_INVALID; }
        R[i] = (float)(x * lc);
        R[i + m] = (float)(y * lc);
        R[i + 2 * m] = (float)(z * lc);
    }
    return RF_OK;
}
