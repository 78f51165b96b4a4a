/*
 * rockfit_b200.h -- C ABI of the B200-native bonded-particle DEM engine.
 *
 * Every entry point returns an rf_status and takes plain pointers, sizes and
 * scalars. Device pointers are CUDA device memory on the current device;
 * host pointers are ordinary host memory. Streams are cudaStream_t passed as
 * an opaque pointer (NULL = the legacy default stream).
 *
 * Two families of entry points:
 *
 *  md_*  -- drop-in replacements for the RockFit-DEM hot-path kernels and step
 *           operations. They work IN PLACE on buffers laid out exactly as the
 *           reference's md_data_types.h lays them out:
 *             particle vectors R, V, W, F, M : float[3N], planes x | y | z at 0, N, 2N
 *             cell arrays  CI[N], CIs[2N] (sorted cell keys, then particle ids),
 *                          pnC[2*CN] (first particle of each cell, then count)
 *             neighbour rows IL[N*K] (uint_fast32_t ids, empty = UINT_FAST32_MAX),
 *                          ILtype[N*K] (uint8: 1 = bond, 0 = contact/none),
 *                          _1d_iL[N*K] (1 / initial bond length),
 *                          Rij, Oijt, Fijn, Fijt, Mijn, Mijt, Mijadd : rf_float3[N*K]
 *           Ids use uint_fast32_t, the reference's own id type, so a caller
 *           built with the same compiler sees the same struct and array sizes.
 *
 *  rf_*  -- the fused engine: a whole quasi-static or explicit test run with its
 *           own device-resident layout (slot-major bond rows, packed particle
 *           vectors, device-side load reduction, CUDA-graph step loop).
 *
 * Units follow the reference (md_phys_constants.h:5-14): length mm, mass mg,
 * time us; stress therefore in units of 1e9 Pa.
 */
#ifndef ROCKFIT_B200_H
#define ROCKFIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rf_status {
    RF_OK = 0,
    RF_ERR_INVALID = 1,        /* bad argument (null pointer, zero size, inconsistent sizes) */
    RF_ERR_CUDA = 2,           /* a CUDA runtime call failed; see rf_last_error_string() */
    RF_ERR_ROW_OVERFLOW = 3,   /* a neighbour row needed more than K slots; rows left unmodified past K */
    RF_ERR_CELL_RANGE = 4,     /* a particle or neighbour cell fell outside the cell grid */
    RF_ERR_NOT_CONVERGED = 5,  /* FIRE reached its iteration limit */
    RF_ERR_CAPACITY = 6,       /* an internal fixed-capacity table (candidate list) overflowed */
    RF_ERR_NO_DEVICE = 7,      /* no usable CUDA device */
    RF_ERR_STATE = 8           /* call made on an engine in the wrong state */
} rf_status;

typedef void* rf_stream;                       /* cudaStream_t */
typedef struct rf_float3 { float x, y, z; } rf_float3;       /* layout of CUDA float3 */
typedef struct rf_uint3 { unsigned int x, y, z; } rf_uint3;  /* layout of CUDA uint3 */
typedef struct rf_double3 { double x, y, z; } rf_double3;    /* layout of CUDA double3 */

#define RF_EMPTY_SLOT ((uint_fast32_t)UINT_FAST32_MAX)

/* Text of the last error raised on this host thread (CUDA error name or argument check). */
const char* rf_last_error_string(void);
/* Library version, and sizeof(uint_fast32_t) the library was built with. */
int rf_version(void);
int rf_id_bytes(void);

/* ------------------------------------------------------------------------ */
/* Scalar state of a test: the numbers md_task_data carries                 */
/* (md_data_types.h:78-323). rf_task_prepare() fills the derived fields with  */
/* the reference's own formulas and type conversions; a caller migrating from */
/* the reference may instead copy them over from its md_task_data.           */
/* ------------------------------------------------------------------------ */

typedef enum rf_test_kind { RF_TEST_UNIAXIAL = 0, RF_TEST_BRAZIL = 1 } rf_test_kind;

typedef struct rf_potential {              /* potential_data, md_data_types.h:146-186 */
    /* inputs */
    double m_E, m_nu, m_Ec, m_Gc, m_ro, b_r, b_d, p_r, p_e, p_mu, p_mur, a_farcut;
    /* derived by potential_data::CalculateParameters (md_data_types.h:153-185) */
    double m_G, b_S, p_V, p_m, b_dd, p_1d_m, p_I, hm_E, hm_G, p_A, aa_farcut,
           Trayleigh, Tsim, dt, D, a, _1d_a, aa, dt_d_m, dt_d_I;
} rf_potential;

typedef struct rf_sample {                 /* sample_data, md_data_types.h:78-122 */
    rf_double3 A_real, B_real, size_real, center_real;
    double Vext;
    rf_float3 L, A, B, axis, center, size, sized2, hidenpoint, spacesize, spacesized2;
    float R0, H0, Vgenmax;
} rf_sample;

typedef struct rf_cells {                  /* cell_data, md_data_types.h:24-56 */
    rf_uint3 Nr;
    uint64_t N;                            /* number of cells CN */
    float a, _1d_a;
    rf_float3 _1d_Nr;
} rf_cells;

typedef struct rf_compression {            /* compression_data, md_data_types.h:188-294 */
    int32_t Loading, Fracture;
    rf_float3 center, size, sized2;
    rf_double3 size_d, center_d;
    float R, RR, Hd2, C, mu, Area, _1d_Area;
    double V, VLoad, Top, Bottom, TopR, BottomR, FractureStress, FractureStrain,
           MinStress, ZeroStress, Stress, Strain, MaxStrain, Size0;
} rf_compression;

typedef struct rf_task {
    rf_test_kind kind;
    uint64_t N;                            /* particles (particle_data::N) */
    uint32_t K;                            /* slots per particle (interaction_list_data::IonP) */
    float acut, aacut;                     /* interaction_list_data::CalculateParameters */
    rf_potential Po;
    rf_sample S;
    rf_cells C;
    rf_compression Compress;
    uint64_t bloks;                        /* additional_data::bloks = N/1024 + 1 */
    double sz0;                            /* result_data::sz0 = Compress.size.z at the start (md_results.cu:21) */
} rf_task;

/*
 * Fill the derived fields of *t from its inputs, following
 *   potential_data::CalculateParameters   md_data_types.h:153-185
 *   sample_data::SetSpaceSizeSi / SetLSi / CalculateParameters   md_data_types.h:86-121
 *   cell_data::CalculateParameters        md_data_types.h:42-55
 *   interaction_list_data::CalculateParameters md_data_types.h:137-143
 *   compression_data::CalculateUParameters / CalculateBParameters md_data_types.h:196-271
 * Inputs: t->kind, t->N, t->K, t->Po (inputs), space_size_si / specimen_size_si
 * (metres, as SetSpaceSizeSi / SetLSi take them), v_load, min_stress, max_strain.
 * cell_a is C.a (the reference sets it to 2 * a_farcut, mp_determineconjgradient.cu:32).
 */
rf_status rf_task_prepare(rf_task* t, const double space_size_si[3], const double specimen_size_si[3],
                          double cell_a, double v_load, double min_stress, double max_strain);

/* compression_data::CompressU / CompressB (md_data_types.h:223-293): advance the platen one step. */
rf_status md_CompressU(rf_task* t, double pressure);
rf_status md_CompressB(rf_task* t, double pressure);

/*
 * SumForcesULoading / SumForcesBLoading (md_results.cu:34-117): reduce the platen
 * partial sums FL[2*nblocks] (host copy), update Stress, Loading, FractureStress,
 * FractureStrain, Fracture. sz0 is R.sz0, Compress.size.z when the run started
 * (md_results.cu:21). curve (may be NULL) receives (strain, stress_bottom,
 * stress_top) when step % dNsave == 0, as R.h_sFL does; *nsaved is advanced.
 */
rf_status md_SumForcesULoading(rf_task* t, const float* h_FL, uint64_t nblocks, uint64_t step,
                               uint64_t dNsave, double sz0, double* curve, uint64_t* nsaved);

/* ------------------------------------------------------------------------ */
/* md_* device step operations (reference layout, in place, on `stream`).    */
/* ------------------------------------------------------------------------ */

/* d_CalculateCellIndex, md_calculate_cell.cu:28-53 */
rf_status md_CalculateCellIndex(const float* R, uint_fast32_t N, uint_fast32_t* CI, float _1d_a,
                                rf_uint3 cN, rf_stream stream);

/* Scratch bytes md_CellDistribution needs for N particles and CN cells. */
size_t md_CellDistributionScratchBytes(uint_fast32_t N, uint_fast32_t CN);

/*
 * CellDistribution, md_cell_distribution.cu:52-101: cell index per particle,
 * stable sort of (cell, id) into CIs, and per-cell (start, count) into pnC
 * (cells without particles get 0, 0). The sort here is a counting sort; its
 * output equals the reference's stable cub radix sort of (CI, 0..N-1).
 * scratch: device buffer of md_CellDistributionScratchBytes(N, CN) bytes.
 */
rf_status md_CellDistribution(const float* R, uint_fast32_t N, uint_fast32_t* CI, uint_fast32_t* CIs,
                              uint_fast32_t* pnC, uint_fast32_t CN, float _1d_a, rf_uint3 cN,
                              void* scratch, size_t scratch_bytes, rf_stream stream);

/*
 * md_CellDistribution without any allocation. No counterpart in the reference: it is
 * for callers that cannot allocate device memory where they bin -- a framework that
 * owns every device byte through its own allocator, or a plugin that is handed only
 * its input and output buffers. Same outputs as md_CellDistribution; the scratch is a
 * fixed array inside this library (cell grids up to 524,287 cells, about 6.3 MB held
 * by every GPU that loads the library, until exit). Larger grids are rejected with
 * RF_ERR_INVALID. The first call on a device (and the first after a cudaDeviceReset)
 * looks up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture. Like every md_* entry
 * point, the call blocks the calling thread until its work on `stream` has finished,
 * because it reads the device status word back. All calls share the one array, so
 * calls whose work overlaps on the GPU (other streams, other host threads) race:
 * serialise them.
 */
rf_status md_CellDistributionNoAlloc(const float* R, uint_fast32_t N, uint_fast32_t* CI, uint_fast32_t* CIs,
                                     uint_fast32_t* pnC, uint_fast32_t CN, float _1d_a, rf_uint3 cN,
                                     rf_stream stream);

/*
 * InteractionListConstruct + d_ConstructInteractionList,
 * md_interaction_list_construction.cu:163-168, md_interaction_list_construct.cu:13-98:
 * clear IL to empty and fill each row from the 8 octant cells in the reference's
 * visiting order. A row that would exceed K slots is cut at K and the call returns
 * RF_ERR_ROW_OVERFLOW (the reference writes past the row).
 */
rf_status md_InteractionListConstruct(const float* R, uint_fast32_t N, const uint_fast32_t* CIs,
                                      const uint_fast32_t* pnC, uint_fast32_t* IL, uint_fast32_t K,
                                      float a, float _1d_a, float aacut, rf_uint3 cN, uint_fast32_t CN,
                                      rf_stream stream);

/*
 * InteractionListReConstructBPM + d_ReConstructInteractionListbpm,
 * md_interaction_list_construction.cu:176-180, md_interaction_list_reconstructbpm.cu:13-46,80-139:
 * add every neighbour within sqrt(aacut) not yet in the row, at the first free slot,
 * as type 0. A full row returns RF_ERR_ROW_OVERFLOW and is left unchanged.
 */
rf_status md_InteractionListReConstructBPM(const float* R, uint_fast32_t N, const uint_fast32_t* CIs,
                                           const uint_fast32_t* pnC, uint_fast32_t* IL, uint8_t* ILtype,
                                           uint_fast32_t K, float a, float _1d_a, float aacut,
                                           rf_uint3 cN, uint_fast32_t CN, rf_stream stream);

/* d_DeleteFarLinks, md_interaction_list_reconstructbpm.cu:141-186 */
rf_status md_DeleteFarLinks(const float* R, uint_fast32_t N, uint_fast32_t* IL, uint8_t* ILtype,
                            float* _1d_iL, rf_float3* Rij, rf_float3* Oijt, rf_float3* Fijn,
                            rf_float3* Fijt, rf_float3* Mijn, rf_float3* Mijt, rf_float3* Mijadd,
                            uint_fast32_t K, float aacut, rf_stream stream);

/* d_ConstructBoundInteractions, md_boundinteractions_construct.cu:35-106 */
rf_status md_ConstructBoundInteractions(const float* R, const float* V, const float* W,
                                        const uint_fast32_t* IL, uint8_t* ILtype, float* _1d_iL,
                                        rf_float3* Rij, rf_float3* Oijt, rf_float3* Fijn, rf_float3* Fijt,
                                        rf_float3* Mijn, rf_float3* Mijt, rf_float3* Mijadd,
                                        uint_fast32_t N, uint_fast32_t K, float aa_create, float b_r,
                                        rf_stream stream);

/* d_CalculateForcesDEM_22 (bond force, moment and break check), md_calculateforcesdem3.cu:424-483 */
rf_status md_CalculateForcesDEM_22(const float* R, const float* V, const float* W,
                                   const uint_fast32_t* IL, uint8_t* ILtype, const float* _1d_iL,
                                   rf_float3* Rij, rf_float3* Oijt, rf_float3* Mijn, rf_float3* Mijt,
                                   float* F, float* M, uint_fast32_t N, uint_fast32_t K, float dt,
                                   float m_E, float m_G, float b_r, float m_Gcritn, float m_Gcritt,
                                   rf_stream stream);

/* d_CalculateForcesDEM_21 (Hertz-Mindlin contacts), md_calculateforcesdem3.cu:338-422 */
rf_status md_CalculateForcesDEM_21(const float* R, const float* V, const float* W,
                                   const uint_fast32_t* IL, uint8_t* ILtype, const float* _1d_iL,
                                   rf_float3* Rij, rf_float3* Oijt, float* F, float* M,
                                   uint_fast32_t N, uint_fast32_t K, float dt, float m_E, float m_G,
                                   float p_A, float m_mu, float m_muroll, float mP, float rP,
                                   rf_stream stream);

/* d_CalculateIncrementsDEM, md_calculateincrementsdem.cu:19-49 */
rf_status md_CalculateIncrementsDEM(const float* F, float* V, float* R, const float* M, float* W,
                                    uint_fast32_t N, float _1d_Mass_m_dt, float dt, float _1d_I_m_dt,
                                    rf_stream stream);

/*
 * d_braziltest_simple2, md_braziltest_simple2.cu:19-151. Platen contact, friction and
 * clamp; the reaction sums go to FL as the reference lays them out: FL[0..nblocks)
 * bottom partials then FL[nblocks..2*nblocks) top partials, so the reference's
 * SumForcesULoading reads the same totals. Here the totals sit in FL[0] and
 * FL[nblocks]; the other partials are 0.
 */
rf_status md_braziltest_simple2(float* R, float* V, float* F, float* FL, uint_fast32_t N,
                                rf_float3 c, float RR, float Yt, float Yb, float Ytr, float Ybr,
                                float vt, float Zcut, uint64_t nblocks, rf_stream stream);

/* d_UniaxialCompression3_simple, md_uniaxialcompression3_simple.cu:19-136 (FL as above) */
rf_status md_UniaxialCompression3_simple(float* R, float* V, float* F, float* FL, uint_fast32_t N,
                                         rf_float3 c, float RR, float Zt, float Zb, float Ztr, float Zbr,
                                         float vt, float Zcut, uint64_t nblocks, rf_stream stream);

/* d_ParallelepipedCutRestriction, md_parallelepipedrestriction.cu:73-159 */
rf_status md_ParallelepipedCutRestriction(float* R, float* V, float* F, uint_fast32_t N,
                                          rf_float3 center, rf_float3 sized2, rf_float3 hp,
                                          rf_stream stream);

/* FIRE pieces, md_firerelaxation.cu:18-70 and :372-490 */
rf_status md_CalculateIncrementsFIRE(const float* F, float* V, float* R, uint_fast32_t N,
                                     float _1d_Mass_m_dt, float dt, float F_alpha, rf_stream stream);
rf_status md_CalculateDecrementsHalfStepFIRE(const float* V, float* R, uint_fast32_t N, float dt_d2,
                                             rf_stream stream);
/* d_FdotVEntire: P = sum_i F_i . V_i as nblocks per-block partial sums (device doubles,
   FdotV[0..nblocks)); the caller adds them in order, as CalculateGPUStepsContractRelaxFIRE
   adds the reference's partials (md_firerelaxation.cu:239-245). */
rf_status md_FdotVEntire(const float* V, const float* F, double* FdotV, uint64_t nblocks, uint_fast32_t N,
                         rf_stream stream);

/* firerelax_data (md_data_types.h:296-301) without its buffers; FdotV is kept in double. */
typedef struct rf_fire {
    uint64_t bloks4, NPpositiveMax, NPnegativeMax, NPpositive, NPnegative, Ndelay, MaxStepsRelaxation;
    float dtmax, dtmin, dt0, dt, alpha0, alpha, dtgrow, dtshrink, alphashrink;
    double FdotV;
} rf_fire;
/* SetFIREData (md_firerelaxation.cu:72-84), plus what CalculateGPUStepsContractRelaxFIRE
   sets before its loop (NPpositive = NPnegative = 0, dt = dt0, :89-91). The reference
   never initialises alpha; here it starts at alpha0. */
rf_status md_SetFIREData(rf_fire* f, uint_fast32_t N, const rf_potential* Po);
/* The host FIRE decision of one relaxation step (md_firerelaxation.cu:266-301) given the
   summed power FdotV: updates NPpositive / NPnegative, dt and alpha. *half_step = 1 when
   the caller must run md_CalculateDecrementsHalfStepFIRE(0.5 * dt) and zero V before the
   increments; *stop = 1 when NPnegative exceeded NPnegativeMax (the loop breaks). */
rf_status md_FireDecide(rf_fire* f, double FdotV, uint64_t step, int* half_step, int* stop);

/* ------------------------------------------------------------------------ */
/* Whole-test drivers (h_CalculationBrazilTest / h_CalculationUniaxialCompression). */
/* ------------------------------------------------------------------------ */

typedef struct rf_run_result {
    uint64_t steps;                /* explicit steps taken */
    double FractureStress, FractureStrain, Stress, Strain;
    int32_t Fracture;
    uint64_t broken_bonds;         /* directed bond slots that broke */
    uint64_t bonds_initial;        /* directed bond slots after bond construction */
    rf_status error;               /* first device-side error seen (RF_OK if none) */
} rf_run_result;

/*
 * h_CalculationBrazilTest / h_CalculationUniaxialCompression
 * (md_calculationbraziltest.cu:113-214, md_calculationuniaxialcompression.cu:113-216):
 * copy h_R in, build cells, rows and bonds, and step until Strain >= MaxStrain,
 * fracture, or max_steps (0 = no limit). t->Compress is updated as the reference
 * updates mdTD.Compress. curve (may be NULL) receives up to curve_cap records of
 * (strain, stress_bottom, stress_top) per step. h_R_out (may be NULL) receives the
 * final positions, float[3N] planar.
 */
rf_status md_CalculationBrazilTest(rf_task* t, const float* h_R, uint64_t max_steps,
                                   double* curve, uint64_t curve_cap, float* h_R_out,
                                   rf_run_result* result);
rf_status md_CalculationUniaxialCompression(rf_task* t, const float* h_R, uint64_t max_steps,
                                            double* curve, uint64_t curve_cap, float* h_R_out,
                                            rf_run_result* result);

/* ------------------------------------------------------------------------ */
/* Fused engine                                                              */
/* ------------------------------------------------------------------------ */

typedef struct rf_engine rf_engine;

/*
 * Create an engine for task *t (prepared) on the current device, copy the
 * particle positions h_R (float[3N] planar, host) in, build rows and bonds
 * (md_calculationbraziltest.cu:132-144). V, W start at zero.
 */
rf_status rf_engine_create(const rf_task* t, const float* h_R, rf_engine** out);

/*
 * Extended model (no reference counterpart: the reference is mono-sized FP32 with
 * global bond constants). Polydisperse particles with FP64 positions; per-particle
 * mass density*4/3*pi*r^3 (density from t->Po: p_m / p_r^3) and inertia 0.4 m r^2;
 * bonds between pairs whose gap |r_ij| - r_i - r_j is below gap_frac * min(r_i, r_j),
 * bond radius bond_lambda * min(r_i, r_j), FP64 rest length, stiffness per area kn
 * (normal) and ks (shear) in place of E/L0 and G/L0, and tensile / shear strengths
 * drawn per unordered pair from Weibull(weibull_m) with scales sigma_c and tau_c.
 * Contacts are the reference's Hertz-Mindlin with equivalent radius and mass. Units
 * are the reference's (mm, mg, microseconds; stress unit 1e9 Pa).
 */
typedef struct rf_ext_params {
    double kn, ks;            /* bond stiffness per area (stress / length) */
    double bond_lambda;       /* bond radius / min(r_i, r_j) */
    double gap_frac;          /* bonding rule */
    double weibull_m;         /* Weibull modulus of both strengths */
    double sigma_c, tau_c;    /* Weibull scales of the tensile and shear strength */
    uint64_t seed;            /* strength stream; a pair draws from (seed, min(i,j), max(i,j)) */
    double post_peak_drop;    /* 0: stop as the reference does (stress below ZeroStress after
                                 loading); d in (0,1): also stop once the stress, after loading,
                                 is below (1 - d) times its peak so far (post-peak load drop) */
    double list_gap;          /* 0: a pair is listed within a_farcut (the reference's rule); g > 0:
                                 within min(a_farcut, r_i + r_j + g), which keeps the rows of small
                                 particles short when the radii span a wide range */
    int32_t ref_mode;         /* 1: the reference's constants in this model (every radius must equal
                                 t->Po.p_r): bonds where the centre distance is below Po.b_d, bond
                                 radius Po.b_r, stiffness per area m_E / L0 and m_G / L0 from each
                                 bond's own rest length, strengths m_Ec and m_Gc, and the bending
                                 moment summed with the reference's extra dt*E/(4 L0) factor
                                 (md_calculateforcesdem3.cu:131-152). The other fields of this
                                 struct but post_peak_drop and list_gap are then ignored. Explicit
                                 steps only. 0: the extended model as described above. */
    int32_t reserved;         /* 0 */
} rf_ext_params;

/* Create an extended-model engine: h_R double[3N] planar (mm), h_radius double[N].
   t is prepared as for rf_engine_create; t->Po.a_farcut must exceed 2 * max radius. */
rf_status rf_engine_create_ext(const rf_task* t, const rf_ext_params* x, const double* h_R,
                               const double* h_radius, rf_engine** out);
/* FP64 positions of an extended-model engine, double[3N] planar (host). */
rf_status rf_engine_positions_f64(rf_engine* e, double* R);

/*
 * A batch of specimens in one engine (extended model, explicit steps; no reference
 * counterpart): nspec specimens of the same test kind, material, time step, slot count
 * and bond stiffness, each with its own geometry, loading, seed and strength
 * distribution (xs[q]), and at least 128 particles. They are laid out side by side along
 * x, each shifted by a whole number of cells with two empty cells between boxes, so
 * they never interact and each evolves exactly as it would alone on the batch's cell
 * grid. One step kernel advances all of them; each specimen keeps its own platens, load
 * reduction, load curve and stop condition (a finished specimen is frozen); the step
 * loop ends when every specimen is done or the step target is reached.
 * h_R[q]: double[3 N_q] planar, h_radius[q]: double[N_q]. Particle q of the batch's
 * arrays (export, rf_engine_positions_f64) are ordered specimen after specimen, with x
 * shifted by the specimen's offset (rf_engine_spec_info).
 */
rf_status rf_engine_create_batch(const rf_task* tasks, const rf_ext_params* xs, const double* const* h_R,
                                 const double* const* h_radius, int nspec, rf_engine** out);
/* Number of specimens of an engine (1 unless made by rf_engine_create_batch). */
int rf_engine_batch_size(rf_engine* e);
/* Specimen spec's first particle, particle count, x offset, and its task as the engine
   runs it (shifted, with the batch's cell grid); any output may be NULL. */
rf_status rf_engine_spec_info(rf_engine* e, int spec, uint64_t* first, uint64_t* count, double* x_offset,
                              rf_task* task);
/* rf_engine_sync / rf_engine_curve for one specimen (steps are the specimen's own). */
rf_status rf_engine_sync_spec(rf_engine* e, int spec, rf_task* t_out, rf_run_result* r_out);
rf_status rf_engine_curve_spec(rf_engine* e, int spec, double* curve, uint64_t cap, uint64_t* n);

/*
 * Quasi-static loading (extended model; no reference counterpart: the reference's FIRE
 * relaxes a sample-preparation potential, md_firerelaxation.cu:85-368). Each load
 * increment advances the loading platen by strain_inc * initial size (0: relax in place)
 * and relaxes the specimen with FIRE (Bitzek et al. 2006) on the conservative part of the
 * bond and contact model, on the device, until the RMS net particle force is at most tol
 * times the mean normal pair force, or max_iter iterations.
 */
typedef struct rf_relax_params {
    double strain_inc;              /* platen advance per increment / initial specimen size */
    double tol;                     /* residual target (1e-6) */
    double dt0, dt_max, dt_min;     /* FIRE steps of the stiffness-scaled dynamics (each particle's
                                       mass is its summed pair stiffness, so the steps are
                                       dimensionless; stable below about 1.4) */
    double alpha0, f_inc, f_dec, f_alpha;
    uint32_t n_delay;
    uint64_t max_iter;              /* FIRE iterations per increment */
} rf_relax_params;
typedef struct rf_relax_result {
    uint64_t iterations;            /* FIRE iterations of this increment */
    int32_t converged;
    double residual;                /* RMS net force / mean normal pair force at exit */
    double mean_force;              /* mean normal pair force (model force units) */
    double stress, strain;          /* platen stress and specimen strain after the increment */
    uint64_t broken_bonds;          /* directed bond slots broken so far */
    rf_status error;
} rf_relax_result;
/* Defaults: strain_inc 2.5e-5, tol 1e-6, dt0 0.1, dt_max 1.0, dt_min 1e-3, alpha0 0.1,
   f_inc 1.1, f_dec 0.5, f_alpha 0.99, n_delay 5, max_iter 200000. */
rf_status rf_relax_default_params(rf_relax_params* p, const rf_task* t);
/* One load increment. warm (device pointer, may be NULL): float[N][6] per-particle
   predicted displacement (x, y, z) and rotation of the increment, applied before FIRE
   (the rotation as the first iteration's angular velocity, rotation / dt0). */
rf_status rf_engine_load_increment(rf_engine* e, const rf_relax_params* p, const float* warm,
                                   rf_relax_result* r);
/* One load increment of every specimen of a batch engine (rf_engine_create_batch; also
   accepts a one-specimen engine). Each specimen's platen advances by strain_inc times its
   own initial size and its relaxation runs on its own FIRE scalars (dt, alpha, positive
   count, convergence); a specimen whose relaxation stopped stays where it is until the
   others stop, so each specimen ends as its run alone would. warm (device, may be NULL):
   float[N][ldw], columns 0-5 as for rf_engine_load_increment, or, with scaled != 0, in
   the warm-start target units of each particle's own specimen. results: one per
   specimen (broken_bonds: the batch's total). No counterpart in the reference: its
   quasi-static path is the north star's FIRE extension, here batched. */
rf_status rf_engine_load_increment_batch(rf_engine* e, const rf_relax_params* p, const float* warm, int ldw,
                                         int scaled, rf_relax_result* results);
/* The last increment's start positions, relaxed displacement and accumulated rotation,
   each double[N][3] (host; any may be NULL): training pairs for the warm start. */
rf_status rf_engine_increment_fields(rf_engine* e, double* x0, double* dx, double* rot);

/*
 * Warm-start features and targets (device buffers; a batch engine's particles each use
 * their own specimen's sizes). Features of each particle for the next increment of size
 * strain_inc, from the last increment's motion: bf16 [rows][64], rows = N rounded up to
 * 128 (padding rows zero). With D = strain_inc * the specimen's initial size:
 *   0-2 displacement / D; 3-5 rotation * r / D; 6 position along the load axis and
 *   7 distance from it, both relative to the specimen's half sizes; 8-55 up to 12
 *   intact bonds in record order: the partner's displacement minus this one's / D
 *   (3) and the bond strain / strain_inc (1); 56 intact bonds / 12; 57 at a platen;
 *   58 one; 59-63 zero.
 * Targets of the last increment, fp32 [N][6]: displacement / D, rotation * r / D.
 */
rf_status rf_engine_warm_features(rf_engine* e, double strain_inc, void* feat);
rf_status rf_engine_warm_targets(rf_engine* e, double strain_inc, float* targets);
/* rf_engine_load_increment with the MLP's output: pred[i * ldp + 0..5] in the units of
   the targets (scaled back to a displacement and rotation before the increment). */
rf_status rf_engine_load_increment_pred(rf_engine* e, const rf_relax_params* p, const float* pred, int ldp,
                                        rf_relax_result* r);
rf_status rf_engine_destroy(rf_engine* e);

/*
 * Homogeneous strain of the specimen (no reference counterpart; the bench and tests use it
 * to start a run in a loaded, damaged state): every particle position x becomes
 * c + (1 + strain[a]) (x - c) along each axis a about the platen box's centre c, the
 * load axis's platens move with it (Strain is updated), and the platen zone's radius
 * grows with the larger lateral strain. Rest lengths, slot state and velocities are kept,
 * so from the next step on the bonds and contacts carry the strain (bonds stretched past
 * their strength break on that step). Each component in (-0.5, 0.5); one specimen only.
 */
rf_status rf_engine_affine_strain(rf_engine* e, const double strain[3]);

/* Advance nsteps explicit steps (stops early, on device, at fracture / max strain). */
rf_status rf_engine_step(rf_engine* e, uint64_t nsteps);
/* Same, with positions uploaded from host first and results read back after:
   the end-to-end path through host buffers. */
rf_status rf_engine_step_host(rf_engine* e, const float* h_R_in, uint64_t nsteps, float* h_R_out);
/* Block until queued work finishes; copy the scalar test state out. */
rf_status rf_engine_sync(rf_engine* e, rf_task* t_out, rf_run_result* r_out);

/*
 * Export the state in the reference layout (host buffers, any may be NULL):
 * R, V, W : float[3N]; IL : uint_fast32_t[N*K]; ILtype : uint8[N*K];
 * _1d_iL : float[N*K]; Rij, Oijt, Mijn, Mijt : rf_float3[N*K].
 */
rf_status rf_engine_export(rf_engine* e, float* R, float* V, float* W, uint_fast32_t* IL,
                           uint8_t* ILtype, float* _1d_iL, rf_float3* Rij, rf_float3* Oijt,
                           rf_float3* Mijn, rf_float3* Mijt);
/* Import full state (reference layout, host buffers, all required) -- resume. */
rf_status rf_engine_import(rf_engine* e, const float* R, const float* V, const float* W,
                           const uint_fast32_t* IL, const uint8_t* ILtype, const float* _1d_iL,
                           const rf_float3* Rij, const rf_float3* Oijt, const rf_float3* Mijn,
                           const rf_float3* Mijt);

/* Copy the load curve recorded so far: up to cap records of (strain, stress_bottom, stress_top). */
rf_status rf_engine_curve(rf_engine* e, double* curve, uint64_t cap, uint64_t* n);

/* Engine counters: [0] steps, [1] candidate-list rebuilds, [2] live bond slots,
   [3] live contact slots, [4] occupied slots; all as of the last sync. */
rf_status rf_engine_counters(rf_engine* e, uint64_t* out, int n);

/* Autotuner (extended model): times `steps` explicit steps with each compiled variant of
   the step kernel (register caps for 8, 6 and 5 resident 128-thread CTAs per SM) on a
   snapshot of the engine's state, restores the state, and keeps the fastest variant
   for the step graph. All variants compute identical results. *choice: CTAs per SM of
   the pick; ms_out[3] (may be NULL): time of each variant for 8, 6, 5. The reference
   model's step has a single variant (choice 6, no timing). Needs a second copy of the
   engine's device memory while it runs. */
rf_status rf_engine_autotune(rf_engine* e, int steps, int* choice, float* ms_out);

/* Kernel launches the engine issues per explicit step when no rebuild runs. */
int rf_engine_launches_per_step(void);
/* The stream the engine launches on (cudaStream_t), for callers that time or order work. */
rf_stream rf_engine_stream(rf_engine* e);
/* Whether the device-driven CUDA graph loop is in use (1) or plain stream launches (0). */
int rf_engine_uses_graph(rf_engine* e);

/* ------------------------------------------------------------------------ */
/* Seeded synthetic specimens                                                */
/* ------------------------------------------------------------------------ */

/*
 * Deterministic seeded specimen: particles of radius p_r on a jittered cubic
 * lattice of spacing 2*p_r*(1+gap_frac), cut to a cylinder (axis z, diameter d,
 * height h) centred at center (mm). jitter is the uniform half-width of the
 * per-coordinate jitter, in units of p_r. The count goes to *n; with R == NULL
 * nothing else is written, otherwise cap must be >= *n and R receives the
 * positions planar (x | y | z at 0, n, 2n). Order is lattice order (x fastest).
 */
rf_status rf_specimen_lattice_cylinder(uint64_t seed, double p_r, double gap_frac, double jitter,
                                       double d, double h, const double center[3],
                                       float* R, uint64_t cap, uint64_t* n);
/* Same, cut to a Brazilian disc: axis z, diameter d, thickness h. */
rf_status rf_specimen_lattice_disc(uint64_t seed, double p_r, double gap_frac, double jitter,
                                   double d, double h, const double center[3],
                                   float* R, uint64_t cap, uint64_t* n);

/*
 * Seeded polydisperse packing on the GPU (the reference generates positions with
 * cuRAND and relaxes a 1/r repulsion, md_createcylindersample.cu:136-343; this
 * generator is its own design). N radii r0 * U[rmin, rmax] (r0 in mm, rmin and rmax
 * relative to it), centres uniform in a cylinder (axis z, height/diameter = aspect)
 * sized for packing fraction phi, then FIRE with a repulsive Hertz contact (spheres and
 * container wall) while the radii grow in stages to their targets, until the largest
 * overlap is below 2e-4 of the smaller radius. Outputs: R double[3N] planar (centred at
 * center, mm), radius double[N] (mm), the container's diameter and height (mm), and the
 * final largest relative overlap. aspect 0.5 gives a Brazilian disc (axis z). Particles
 * are numbered in spatial order (cells of 6 r0, x fastest, then y, then z), which keeps
 * neighbours close in memory.
 */
rf_status rf_pack_cylinder(uint64_t seed, uint64_t N, double r0, double rmin, double rmax, double aspect,
                           double phi, const double center[3], double* R, double* radius,
                           double* diameter, double* height, double* max_overlap);
/* Radius distributions of rf_pack_cylinder_dist. */
typedef enum rf_radius_dist {
    RF_RADII_UNIFORM = 0,       /* r0 * U[rmin, rmax] (rf_pack_cylinder) */
    RF_RADII_LOG_UNIFORM = 1    /* r0 * rmin * (rmax / rmin)^U[0, 1] */
} rf_radius_dist;
/* rf_pack_cylinder with a choice of radius distribution. */
rf_status rf_pack_cylinder_dist(uint64_t seed, uint64_t N, double r0, double rmin, double rmax, int dist,
                                double aspect, double phi, const double center[3], double* R, double* radius,
                                double* diameter, double* height, double* max_overlap);

/* ------------------------------------------------------------------------ */
/* State files                                                               */
/* ------------------------------------------------------------------------ */

/*
 * The reference's binary state dump, byte for byte: SaveAllData / LoadAllData
 * (md_savealldata.cpp:12-91; write_sample_data :98-111, write_particle_data :127-142,
 * write_interaction_list_data :176-199). id_bytes is the width of uint_fast32_t in the
 * build that reads or wrote the file: 4 for the reference's own (MSVC) build, 8 for a
 * Linux build. The sample's R0 and H0 are written as three floats each, as the
 * reference does: (R0, H0, Vgenmax) and (H0, Vgenmax, the 4 bytes after Vgenmax, which
 * hold the sample's PN with 4-byte ids and padding (0 here) with 8-byte ids). Arrays in
 * the reference layout: F, V, R, M, W float[3N] planar, Q float[4N], IL, ILtype,
 * _1d_iL [N*K], the slot vectors rf_float3[N*K]; a NULL array is written as zeros
 * (R, IL and ILtype are required).
 */
rf_status rf_save_all_data(const char* path, int id_bytes, const rf_sample* S, uint64_t pn, uint64_t N, uint32_t K,
                           float acut, const float* F, const float* V, const float* R, const float* M,
                           const float* W, const float* Q, const uint_fast32_t* IL, const uint8_t* ILtype,
                           const float* _1d_iL, const rf_float3* Rij, const rf_float3* Oijt, const rf_float3* Fijn,
                           const rf_float3* Fijt, const rf_float3* Mijn, const rf_float3* Mijt,
                           const rf_float3* Mijadd);
/* Read a file of rf_save_all_data / SaveAllData. Call with R == NULL to learn N and K
   (and S, pn, acut), then again with buffers of those sizes (NULL arrays other than R,
   IL, ILtype are skipped). Like LoadAllData, S's real extents (A_real, B_real,
   size_real, center_real) are recomputed from the loaded positions. */
rf_status rf_load_all_data(const char* path, int id_bytes, rf_sample* S, uint64_t* pn, uint64_t* N, uint32_t* K,
                           float* acut, float* F, float* V, float* R, float* M, float* W, float* Q,
                           uint_fast32_t* IL, uint8_t* ILtype, float* _1d_iL, rf_float3* Rij, rf_float3* Oijt,
                           rf_float3* Fijn, rf_float3* Fijt, rf_float3* Mijn, rf_float3* Mijt, rf_float3* Mijadd);
/* LAMMPS data text of SaveLammpsDATASimple (md_savelammpsdata.cpp:8-74): box and atoms in
   metres, per-atom translational / rotational / total kinetic energy in joules (zeros
   unless with_energy), one bond line per directed bond slot. */
rf_status rf_save_lammps_data(const char* path, const rf_task* t, uint64_t N, uint32_t K, const float* R,
                              const float* V, const float* W, const uint_fast32_t* IL, const uint8_t* ILtype,
                              int with_energy);
/*
 * Particle positions as text, the reference's sample files (SaveParticleDATAtxt /
 * LoadParticleDATAtxt, md_createcylindersample.cu:104-133): the particle count on the first
 * line, then "x y z" per particle in metres (float mm times 1e-3 as a double, the stream's
 * default 6 significant digits). R is float[3n] planar in mm. Loading: call with R == NULL
 * to learn n, then with cap >= n (RF_ERR_CAPACITY otherwise).
 */
rf_status rf_save_positions_txt(const char* path, const float* R, uint64_t n);
rf_status rf_load_positions_txt(const char* path, float* R, uint64_t cap, uint64_t* n);

/*
 * Versioned checkpoint of a reference-model engine: a header ("RFB2CKPT", version 1, id
 * width, the rf_task as rf_engine_sync returns it) followed by the rf_save_all_data
 * payload of the engine's exported state. rf_engine_restore makes an engine from such a
 * file whose steps continue the saved run bit for bit (the load curve restarts).
 */
rf_status rf_engine_checkpoint(rf_engine* e, const char* path);
rf_status rf_engine_restore(const char* path, rf_engine** out);

/* ------------------------------------------------------------------------ */
/* BF16 tensor-core GEMM (tcgen05, FP32 accumulation in tensor memory) and the */
/* warm-start MLP. No reference counterpart.                                  */
/* ------------------------------------------------------------------------ */

/* Epilogues of rf_gemm_bf16. */
typedef enum rf_gemm_epilogue {
    RF_EPI_RELU_BF16 = 0,   /* out_h = bf16(relu(acc + bias)), out_ht = its transpose (optional) */
    RF_EPI_LINEAR_F32 = 1,  /* out_f = (acc + bias) * scale, first ncols_f columns */
    RF_EPI_MASK_BF16 = 2,   /* out_h = bf16(mask > 0 ? acc : 0) (+ transpose): ReLU backward */
    RF_EPI_ATOMIC_F32 = 3   /* out_f += scale * acc (split-K over `splits` CTAs) */
} rf_gemm_epilogue;
/*
 * C[M x N] = A[M x K] * B[N x K]^T on the device. A, B: bf16, row-major with K
 * contiguous (leading dimensions lda, ldb in elements, multiples of 8; 16-byte aligned
 * bases); N a multiple of 16 up to 256; K a multiple of 8. bias: float[N] or NULL;
 * mask: bf16 [M x ldm]. Outputs as the epilogue says; out_ht is [N x ld_ht] (ld_ht >= M).
 * Asynchronous on `stream`; rf_gemm_status reports a tensor-core wait that timed out.
 */
rf_status rf_gemm_bf16(const void* A, int lda, const void* B, int ldb, int M, int N, int K, int mode,
                       const float* bias, const void* mask, int ldm, void* out_h, int ld_h, void* out_ht,
                       int ld_ht, float* out_f, int ld_f, int ncols_f, float scale, int splits,
                       rf_stream stream);
rf_status rf_gemm_status(rf_stream stream);

/*
 * Warm-start MLP (per particle): 64 features -> 128 -> 128 -> 128 -> 6, ReLU, BF16
 * weights and activations, FP32 accumulation on the tensor cores, FP32 master weights
 * trained with Adam on mean((y - t)^2). Layer l's weights W[l] are [out][in] (the last
 * layer stored as 16 x 128, rows 6..15 zero).
 */
typedef struct rf_mlp rf_mlp;
rf_status rf_mlp_create(uint64_t seed, rf_mlp** out);
rf_status rf_mlp_destroy(rf_mlp* m);
rf_stream rf_mlp_stream(rf_mlp* m);
/* Y[rows][ldy] (first ncols <= 16 outputs, fp32, device) from X (bf16 [rows][64], device). */
rf_status rf_mlp_forward(rf_mlp* m, const void* X, int rows, float* Y, int ldy, int ncols);
/* One training step on X (bf16 [rows][64]) and targets T (fp32 [rows][6]), both on the
   device: loss before the step into *loss; an Adam step with rate lr when lr > 0. */
rf_status rf_mlp_train_step(rf_mlp* m, const void* X, const float* T, int rows, float lr, double* loss);
/* Residual mode: outputs are x[0:6] + network(x), i.e. the network learns the correction
   to the last increment's motion (features 0-5). Off by default. */
rf_status rf_mlp_set_residual(rf_mlp* m, int on);
/* Host copies of layer `layer`'s fp32 weights / bias, and of the last step's gradients
   (gT is [in][out]). */
rf_status rf_mlp_get(rf_mlp* m, int layer, float* W, float* b);
rf_status rf_mlp_set(rf_mlp* m, int layer, const float* W, const float* b);
rf_status rf_mlp_grad(rf_mlp* m, int layer, float* gT, float* gb);

#ifdef __cplusplus
}
#endif
#endif /* ROCKFIT_B200_H */
