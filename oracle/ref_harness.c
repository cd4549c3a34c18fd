/*
 * Test infrastructure (oracle): a harness around the reference mini-app's own
 * C sources, compiled from where they lie by oracle/Makefile.  Nothing here is
 * on the product path; tests, the golden-fixture script and bench.py's
 * reference arm load the resulting oracle/_ref/libswe_ref_*.so through ctypes.
 *
 * It owns the globals that the reference's main.c defines (main.c:33-40:
 * sim_params, LPSMD, local_timer, mpi_rank, mpi_size) and replays main.c's
 * initialisation sequence (main.c:90-179): binary read, optional RCM reorder,
 * padding, SFDL conversion, H tiling for non-CFDL builds, patch decomposition
 * and the serial LPSMD copy.  The time step itself is the reference's own
 * RK_substep / eval_RHS_swe (swe_code/main/rk4_rbffd_swe.c:30-72, :189-362).
 */
#include <swe_config.h>
#include <input.h>
#include <rcm.h>
#include <reorder_nodes.h>
#include <layout.h>
#include <matrix_transformations.h>
#include <init_patches.h>
#include <rk4_rbffd_swe.h>
#include <profiling.h>

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* Globals owned by the reference's main.c (main.c:33-40). */
sim_params_struct sim_params;
PSMD_struct* LPSMD;
timing_struct local_timer;
int mpi_rank;
int mpi_size;

/* reference: rk4_rbffd_swe.c:189 (external linkage, not in a header) */
void eval_RHS_swe(fType* K, fType* F);

static fType* g_H_init = NULL;
static fType* g_H_100 = NULL;
static int* g_mapping = NULL;
static int g_Nnodes = 0;
static int g_loaded = 0;

#define REFH_LAYOUT_CFDL 1
#define REFH_LAYOUT_SFDL 2

static int layout_flags(void) {
    int f = 0;
#ifdef USE_CFDL
    f |= REFH_LAYOUT_CFDL;
#endif
#ifdef USE_SFDL
    f |= REFH_LAYOUT_SFDL;
#endif
    return f;
}

/* Replays main.c:90-179 for one serial rank.  Returns 0 on success.  May be
 * called again with another file; the previous arrays are leaked, as the
 * reference never frees them either. */
int refh_load(const char* path, int use_rcm) {
    mpi_rank = 0;
    mpi_size = 1;
    memset(&sim_params, 0, sizeof(sim_params));
    strncpy(sim_params.inputFile, path, MAX_FILE_PATH_SIZE - 1);
    sim_params.nsteps = 1;
    sim_params.nattempts = 1;
    sim_params.USE_RCM = use_rcm;
    local_timer = init_timer(1);
    local_timer.attempt = 0;

    LPSMD = (PSMD_struct*)malloc(sizeof(PSMD_struct));
    GSMD_struct GSMD = get_GSMD_bin(sim_params.inputFile);
    fType* H_init_global = get_ICs_bin(sim_params.inputFile);
    fType* H_100_global = get_FCs_bin(sim_params.inputFile);
    g_Nnodes = GSMD.Nnodes;

    g_mapping = (int*)malloc(sizeof(int) * GSMD.Nnodes);
    if (use_rcm == 1) {
        int* mapping = rcm_mapping(GSMD);
        memcpy(g_mapping, mapping, sizeof(int) * GSMD.Nnodes);
        GSMD = reorder_GSMD_struct(mapping, GSMD);
        H_init_global = reorder_2D_fp_arr(H_init_global, mapping, GSMD.Nnodes, 4);
        H_100_global = reorder_2D_fp_arr(H_100_global, mapping, GSMD.Nnodes, 4);
        free(mapping);
    } else {
        for (int i = 0; i < GSMD.Nnodes; i++) g_mapping[i] = i;
    }

    GSMD = pad_GSMD_data(GSMD);
    H_init_global = pad_2D_fp_arr(H_init_global, GSMD.Nnodes, GSMD.padded_Nnodes, 4, 4);
    H_100_global = pad_2D_fp_arr(H_100_global, GSMD.Nnodes, GSMD.padded_Nnodes, 4, 4);
#ifdef USE_SFDL
    GSMD = convert2_SFDL(GSMD);
#endif
#ifndef USE_CFDL
    H_init_global = transpose_2D_fp_arr(H_init_global, GSMD.padded_Nnodes, 4);
    H_init_global = tile_2D_fp_arr(H_init_global, 4, GSMD.padded_Nnodes, SIMD_LENGTH);
    H_100_global = transpose_2D_fp_arr(H_100_global, GSMD.padded_Nnodes, 4);
    H_100_global = tile_2D_fp_arr(H_100_global, 4, GSMD.padded_Nnodes, SIMD_LENGTH);
#endif
    patch_struct* GPD = get_GPD(GSMD);
    init_LPSMD(GPD, GSMD);
    g_H_init = get_patch_ICs(H_init_global, GPD);
    g_H_100 = get_patch_ICs(H_100_global, GPD);
    g_loaded = 1;
    return 0;
}

/* info[0..8] = patch_size, compute_size, Nnbr, padded_Nnbr, sizeof(fType),
 * layout flags (1 = CFDL, 2 = SFDL), SIMD_LENGTH, compute_pid_s, Nnodes. */
void refh_info(int* info) {
    info[0] = LPSMD->patch_size;
    info[1] = LPSMD->compute_size;
    info[2] = LPSMD->Nnbr;
    info[3] = LPSMD->padded_Nnbr;
    info[4] = (int)sizeof(fType);
    info[5] = layout_flags();
    info[6] = SIMD_LENGTH;
    info[7] = LPSMD->compute_pid_s;
    info[8] = g_Nnodes;
}

/* build-time facts, available before refh_load */
int refh_fsize(void) { return (int)sizeof(fType); }
int refh_layout(void) { return layout_flags(); }
int refh_simd_length(void) { return SIMD_LENGTH; }

const PSMD_struct* refh_psmd(void) { return LPSMD; }
double refh_gh0(void) { return (double)LPSMD->gh0; }
double refh_dt(void) { return (double)LPSMD->dt; }
const fType* refh_H_init(void) { return g_H_init; }
const fType* refh_H_100(void) { return g_H_100; }
const int* refh_mapping(void) { return g_mapping; }

/* Static arrays of LPSMD, by name, for tests that inspect the layouts. */
const void* refh_array(const char* name) {
    if (!strcmp(name, "x")) return LPSMD->x;
    if (!strcmp(name, "y")) return LPSMD->y;
    if (!strcmp(name, "z")) return LPSMD->z;
    if (!strcmp(name, "f")) return LPSMD->f;
    if (!strcmp(name, "ghm")) return LPSMD->ghm;
    if (!strcmp(name, "p_u")) return LPSMD->p_u;
    if (!strcmp(name, "p_v")) return LPSMD->p_v;
    if (!strcmp(name, "p_w")) return LPSMD->p_w;
    if (!strcmp(name, "gradghm")) return LPSMD->gradghm;
    if (!strcmp(name, "idx")) return LPSMD->idx;
    if (!strcmp(name, "Dx")) return LPSMD->Dx;
    if (!strcmp(name, "Dy")) return LPSMD->Dy;
    if (!strcmp(name, "Dz")) return LPSMD->Dz;
    if (!strcmp(name, "L")) return LPSMD->L;
    return NULL;
}

/* reference eval_RHS_swe on caller buffers (K: patch_size*4, F: compute_size*4) */
void refh_eval_rhs(fType* K, fType* F) { eval_RHS_swe(K, F); }

/* reference RK_substep on caller buffers */
void refh_rk_substep(fType* H, fType* K, fType* F, fType* D, int substep_id) {
    RK_substep(H, K, F, D, substep_id);
}

/* Runs nsteps full RK4 steps of the reference on H in place (main.c:336-358)
 * and returns the wall-clock seconds of the loop.  eval_rhs_seconds receives
 * the reference's own accumulated eval_RHS_swe timer for the same loop. */
double refh_run(fType* H, int nsteps, double* eval_rhs_seconds) {
    fType* K = (fType*)malloc(sizeof(fType) * LPSMD->patch_size * 4);
    fType* F = (fType*)malloc(sizeof(fType) * LPSMD->compute_size * 4);
    fType* D = (fType*)malloc(sizeof(fType) * LPSMD->compute_size * 4);
    memcpy(K, H, sizeof(fType) * LPSMD->patch_size * 4);
    local_timer.attempt = 0;
    local_timer.t_eval_rhs[0] = 0.0;
    double t0 = getTime();
    for (int s = 1; s <= nsteps; s++)
        for (int rk = 0; rk < 4; rk++) RK_substep(H, K, F, D, rk);
    double t = getTime() - t0;
    if (eval_rhs_seconds) *eval_rhs_seconds = local_timer.t_eval_rhs[0];
    free(K);
    free(F);
    free(D);
    return t;
}

/* Element-wise |H - H_100| > TOLERANCE (or NaN) count over the compute range,
 * the same test as verify_output (main.c:439-477). */
int refh_verify(const fType* H, double* max_abs_err) {
    int count = 0;
    double mx = 0.0;
    for (int i = LPSMD->compute_pid_s; i < LPSMD->compute_pid_e; i++) {
        for (int j = 0; j < 4; j++) {
            fType d = H[SVM_LIN_ID(i, j)] - g_H_100[SVM_LIN_ID(i, j)];
            d = d < 0 ? -d : d;
            if (d > TOLERANCE || d != d) count++;
            if ((double)d > mx || d != d) mx = (double)d;
        }
    }
    if (max_abs_err) *max_abs_err = mx;
    return count;
}

double refh_tolerance(void) { return (double)TOLERANCE; }
