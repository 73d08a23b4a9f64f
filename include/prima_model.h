/* prima_model.h -- the host-side model layer in front of the device solve:
 * the MPS reader and the exact presolve, in C++ inside libprima_cuda.so.
 *
 * Reference interfaces replaced:
 *   prima_mps_*      MpsReader.read / MpsReader.fromLines and MpsInstance
 *                    (modules/prima-mps/src/main/scala/org/noaidi/prima/mps/
 *                    MpsReader.scala:14-32, :62-81, :91-235)
 *   prima_presolve*  Presolve.apply / PresolveResult.restore
 *                    (modules/prima-core/src/main/scala/org/noaidi/prima/
 *                    Presolve.scala:65-191, :199-408)
 *
 * Neither needs a GPU.  Every call returns PRIMA_OK or an error code;
 * prima_last_error() gives the message.  A malformed file is
 * PRIMA_ERR_PARSE (MpsParseException); a model the LP builder refuses is
 * PRIMA_ERR_INVALID_ARGUMENT (the reference's `require`).  Handles own their
 * arrays; prima_lp views obtained from them stay valid until the handle is
 * freed. */
#ifndef PRIMA_MODEL_H
#define PRIMA_MODEL_H

#include "prima_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- MPS (MpsReader.scala) --------------------------------------------- */

typedef struct prima_mps_instance prima_mps_instance;

/* MpsReader.fromLines over a text buffer of `length` bytes; `fallback_name`
 * names the instance when the file has no NAME line. */
int32_t prima_mps_read(const char *text, int64_t length, const char *fallback_name, prima_mps_instance **out);
/* MpsReader.read(path): the file's base name is the fallback name. */
int32_t prima_mps_read_file(const char *path, prima_mps_instance **out);
void prima_mps_free(prima_mps_instance *mps);

typedef struct {
  int32_t num_variables;   /* columns, in order of first appearance */
  int32_t num_constraints; /* standard-form rows */
  int32_t num_equalities;
  int32_t num_rows;        /* constraint rows as the file declares them */
  int64_t nnz;
  int32_t num_integer_columns;
  int32_t pad;
} prima_mps_info;

int32_t prima_mps_get_info(const prima_mps_instance *mps, prima_mps_info *info);
/* The standard-form LpProblem (LpBuilder.build, LpProblem.scala:209-248). */
int32_t prima_mps_get_problem(const prima_mps_instance *mps, prima_lp *lp);
/* RowTranslation (LpProblem.scala:152-207), per declared row:
 * kind 0 direct (row first), 1 negated (row first), 2 range (lower row
 * first, upper row second); `second` is -1 unless kind is 2. */
int32_t prima_mps_get_translation(const prima_mps_instance *mps, int32_t *kind, int32_t *first, int32_t *second);
const char *prima_mps_name(const prima_mps_instance *mps);
const char *prima_mps_row_name(const prima_mps_instance *mps, int32_t row);
const char *prima_mps_column_name(const prima_mps_instance *mps, int32_t column);
/* Integer columns (MARKER blocks, BV, LI, UI), ascending. */
int32_t prima_mps_get_integer_columns(const prima_mps_instance *mps, int32_t *columns);

/* ---- presolve (Presolve.scala) ------------------------------------------ */

typedef struct prima_presolved prima_presolved;

typedef struct {
  int32_t fixed_columns;         /* Presolve.Stats (Presolve.scala:50-62) */
  int32_t empty_columns;
  int32_t empty_rows;
  int32_t singleton_rows;
  int32_t proven_infeasible;     /* the only status presolve proves */
  int32_t unbounded_if_feasible; /* an empty column's cost points at an infinite bound */
  int32_t passes;
  int32_t reduced_variables;
  int32_t reduced_constraints;
  int32_t reduced_equalities;
  int64_t reduced_nnz;
} prima_presolve_info;

/* Presolve.apply: fixed columns, empty rows, singleton rows and empty
 * columns, in passes until nothing changes or `max_passes` (20 in the
 * reference) is reached.  The input is copied. */
int32_t prima_presolve(const prima_lp *lp, int32_t max_passes, prima_presolved **out);
void prima_presolve_free(prima_presolved *presolved);
int32_t prima_presolve_get_info(const prima_presolved *presolved, prima_presolve_info *info);
/* The reduced LpProblem; PRIMA_ERR_INVALID_ARGUMENT when presolve proved
 * infeasibility (there is nothing to solve). */
int32_t prima_presolve_get_reduced(const prima_presolved *presolved, prima_lp *reduced);
/* Original index of each reduced column and row. */
int32_t prima_presolve_get_maps(const prima_presolved *presolved, int32_t *column_map, int32_t *row_map);
/* PresolveResult.restore's vector part: a reduced solution's primal, dual
 * and reduced costs mapped back to the original problem, singleton rows
 * priced from the reduced cost of the column they bound, fixed columns'
 * reduced costs c - K'y from the restored duals. */
int32_t prima_presolve_restore(const prima_presolved *presolved, const double *primal, const double *dual,
                               const double *reduced_costs, double *primal_out, double *dual_out,
                               double *reduced_costs_out);

#ifdef __cplusplus
}
#endif

#endif /* PRIMA_MODEL_H */
