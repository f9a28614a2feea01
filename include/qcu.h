/*
 * qcu.h - drop-in C interface of the B200 Wilson-clover solver.
 *
 * Same types, names, signatures and argument meaning as the reference's
 * public header (YellowBicycleee/Qcu_Cg_Inverter, cg_inverter/include/qcu.h:1-25)
 * so that an existing caller can relink against libqcu_b200.so unchanged.
 * All field pointers are DEVICE pointers owned by the caller, in the
 * reference's AoS layouts (complex double):
 *   gauge        [dir 4][parity 2][t][z][y][x/2][3][3]
 *   half spinor  [t][z][y][x/2][spin 4][colour 3]
 *   full spinor  [parity 2][half spinor]       (even sites first)
 * The calls are synchronous on return, like the reference's.
 *
 * Differences that a caller can observe, all in the caller's favour:
 *  - errors never call exit(): the call returns early and qcu_last_error()
 *    reports a code (the reference prints and exits, include/qcu_macro.cuh:34-41);
 *  - loadQcuGauge() and initGridSize() invalidate the cached clover term (the
 *    reference computes it once per process and never again,
 *    src/qcu_clover_dslash.cu:564-566, 794-825);
 *  - lattices need not have a half volume divisible by 256
 *    (src/qcu_clover_dslash.cu:866-868 truncates the grid); only Lx even is required.
 */
#ifndef QCU_H
#define QCU_H

#ifdef __cplusplus
extern "C" {
#endif

/* reference: include/qcu.h:7-9 - lattice extent (x, y, z, t) of this rank */
typedef struct QcuParam_s {
  int lattice_size[4];
} QcuParam;

/* reference: include/qcu.h:11-13 - process grid; only {1,1,1,1} is accepted */
typedef struct QcuGrid_t {
  int grid_size[4];
} QcuGrid_t;

/* reference: include/qcu.h:14, src/qcu_communicator.cu:1630-1650.
 * Must be called first. Creates the library context for this lattice on the
 * current device and remembers `gauge`. A grid other than {1,1,1,1} is
 * rejected with QCU_ERR_UNSUPPORTED (this build runs on one GPU). */
void initGridSize(QcuGrid_t* grid, QcuParam* p_param, void* gauge, void* fermion_in, void* fermion_out);

/* reference: include/qcu.h:15, src/dslash.cu:62-77.
 * fermion_out (half spinor of `parity`) = D fermion_in (half spinor of
 * 1-parity): the Wilson hopping term without kappa, periodic boundaries. */
void dslashQcu(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int parity);

/* reference: include/qcu.h:17, src/dslash.cu:78-80 -> src/qcu_clover_dslash.cu:948-987.
 * Full spinors: fermion_out = (A - D) fermion_in, or (A - D^dag) when
 * dagger_flag != 0, with the reference normalisation kappa = kappa*c_sw = 1. */
void fullDslashQcu(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int dagger_flag);

/* reference: include/qcu.h:18, src/cg_inverter.cu:260-369.
 * x_vector <- solution for the source b_vector (full spinors), by the
 * reference's own CG flow on (1 - A^-1 D^dag)(1 - A^-1 D) (complex alpha and
 * beta, stop when |<r,r>| < 1e-23, at most V iterations). */
void cg_inverter(void* b_vector, void* x_vector, void* gauge, QcuParam* param);

/* reference: include/qcu.h:20, src/dslash.cu:27-35.
 * Reads the AoS gauge field and keeps it resident in the internal layout
 * (double, single and 16-bit copies). */
void loadQcuGauge(void* gauge, QcuParam* param);

/* reference: include/qcu_clover_dslash.cuh:24, src/qcu_clover_dslash.cu:902-919
 * (C++ linkage there; exported here with C linkage and also under the
 * reference's C++ symbol name). Like the reference, it applies A^-1 IN PLACE
 * to fermion_out (full spinor) and ignores fermion_in. */
void invertCloverDslash(void* fermion_out, void* fermion_in, void* gauge, QcuParam* param, int invert_flag);

/* Status of the last call made by this thread through either header
 * (0 = success; codes in qcu_b200.h). No counterpart in the reference, which
 * has no error reporting. */
int qcu_last_error(void);
const char* qcu_last_error_string(void);

#ifdef __cplusplus
}
#endif
#endif
