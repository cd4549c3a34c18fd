/*
 * Test infrastructure (oracle): forced configuration header for building the
 * reference mini-app's C sources in FP64.
 *
 * The reference hard-defines RUN_32BIT in swe_code/main/include/swe_config.h:75,
 * so its sources always build with fType = float.  Its FP64 mode
 * (swe_config.h:84-89: fType = double, TOLERANCE 1e-9) is only reachable by
 * editing that line.  Instead of editing or copying the reference, the oracle
 * recipe force-includes this header (gcc -include) ahead of every reference
 * translation unit.  It defines the reference's include guard SWE_CONFIG_H, so
 * the reference header is skipped, and restates the same macros and struct
 * layouts with fType = double.
 *
 * The macros and structs below must stay member-for-member identical to
 * swe_config.h:17-279 (they are an ABI shared with the reference sources);
 * only the RUN_32BIT switch differs.
 */
#ifndef SWE_CONFIG_H
#define SWE_CONFIG_H

#ifndef SIMD_LENGTH
#define SIMD_LENGTH 8
#endif

/* swe_config.h:21-22 */
#define ROUNDUP_SIMD(N) (((((N) - 1) / SIMD_LENGTH) + 1) * SIMD_LENGTH)
#define ROUNDDOWN_SIMD(N) (((N) / SIMD_LENGTH) * SIMD_LENGTH)

/* swe_config.h:31-37: differentiation-matrix and 3-vector linear ids */
#ifdef USE_SFDL
#define DM_LIN_ID(NODE_ID, NBR_ID, NNBR) \
    ((ROUNDDOWN_SIMD(NODE_ID) * (NNBR)) + ((NBR_ID) * SIMD_LENGTH) + ((NODE_ID) % SIMD_LENGTH))
#define VECT_LIN_ID(NODE_ID, COMP_ID) \
    ((ROUNDDOWN_SIMD(NODE_ID) * 3) + ((COMP_ID) * SIMD_LENGTH) + ((NODE_ID) % SIMD_LENGTH))
#else
#define DM_LIN_ID(NODE_ID, NBR_ID, NNBR) (((NODE_ID) * (NNBR)) + (NBR_ID))
#define VECT_LIN_ID(NODE_ID, COMP_ID) (((NODE_ID) * 3) + (COMP_ID))
#endif

#define X_COMP_ID 0
#define Y_COMP_ID 1
#define Z_COMP_ID 2

/* swe_config.h:50-54: state-variable-matrix linear id */
#ifdef USE_CFDL
#define SVM_LIN_ID(PID, SV_ID) ((4 * (PID)) + (SV_ID))
#else
#define SVM_LIN_ID(PID, SV_ID) \
    ((ROUNDDOWN_SIMD(PID) * 4) + ((SV_ID) * SIMD_LENGTH) + ((PID) % SIMD_LENGTH))
#endif

#define U_SV_ID 0
#define V_SV_ID 1
#define W_SV_ID 2
#define H_SV_ID 3

#define MAX_FILE_PATH_SIZE 200

typedef double fType_Input;
/* FP64 model precision: the branch swe_config.h:84-89 selects when RUN_32BIT is absent */
typedef double fType;
#define TOLERANCE 1.0e-9

typedef struct sim_params_struct {
    char inputFile[MAX_FILE_PATH_SIZE];
    int nsteps;
    int nattempts;
    int num_compute_units;
    int USE_NETCDF;
#ifdef USE_HIST
    char outputFile[MAX_FILE_PATH_SIZE];
    int history_interval;
#endif
    int USE_RCM;
    int OCL;
} sim_params_struct;

typedef struct GSMD_struct {
    int Nnodes, padded_Nnodes;
    fType* x;
    fType* y;
    fType* z;
    fType* f;
    fType g;
    fType a;
    fType gh0;
    fType dt;
    fType* ghm;
    fType* gradghm;
    fType* p_u;
    fType* p_v;
    fType* p_w;
    int Nnbr, padded_Nnbr;
    fType gamma;
    int* idx;
    fType* Dx;
    fType* Dy;
    fType* Dz;
    fType* L;
} GSMD_struct;

typedef struct patch_struct {
    int halo_gid_s;
    int halo_gid_e;
    int compute_gid_s;
    int compute_gid_e;
    int lnbr_halo_gid_e;
    int rnbr_halo_gid_s;
    int compute_size;
    int patch_size;
} patch_struct;

typedef struct PSMD_struct {
    int lnbr_rank;
    int rnbr_rank;
    int patch_size, compute_size, lhalo_size, rhalo_size;
    int halo_pid_s, compute_pid_s, compute_pid_e, halo_pid_e;
    int lnbr_halo_size, rnbr_halo_size;
    int lnbr_halo_pid_e, rnbr_halo_pid_s;
    fType* x;
    fType* y;
    fType* z;
    fType* f;
    fType gh0;
    fType dt;
    fType* ghm;
    fType* gradghm;
    fType* p_u;
    fType* p_v;
    fType* p_w;
    int Nnbr, padded_Nnbr;
    int* idx;
    fType* Dx;
    fType* Dy;
    fType* Dz;
    fType* L;
} PSMD_struct;

typedef struct timing_struct {
    int attempt;
    double t_init;
    double t_ocl;
    double* t_main;
    double* t_eval_rhs;
    double* t_mpi;
    double* t_eval_K;
    double* t_update_D;
    double* t_update_H;
} timing_struct;

#endif
