/* CPU oracle for the KushDB hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A row-at-a-time restatement of the reference's generated-code semantics for
 * ScanSelect / Select / HashJoin / GroupByAggregate / Aggregate / OrderBy /
 * SkinnerJoin / Output, used by the tests, the smoke check and the CPU
 * baseline leg of the benchmark to check the GPU engine.  The product path
 * never links or calls it.  Its parity with the reference is pinned by the
 * reference's golden tables (tests/golden/), see oracle.cc for the per-rule
 * file:line citations.
 */
#ifndef KDB_ORACLE_H_
#define KDB_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kdbo_ctx kdbo_ctx;
typedef struct kdbo_result kdbo_result;

kdbo_ctx* kdbo_create(void);
void kdbo_destroy(kdbo_ctx* ctx);
const char* kdbo_last_error(kdbo_ctx* ctx);

/* Fixed-width column: `data` holds n values of the type's width (int8 for
 * BOOLEAN, int16 SMALLINT, int32 INT/DATE/ENUM, int64 BIGINT, f64 REAL).
 * `nulls` (may be NULL) holds n int8 flags, 1 = NULL.  Data is copied. */
int kdbo_register_column(kdbo_ctx* ctx, const char* table, const char* column,
                         const char* type, const void* data, int64_t n,
                         const int8_t* nulls);
/* TEXT column: value r is chars[offsets[r] .. offsets[r+1]). */
int kdbo_register_text_column(kdbo_ctx* ctx, const char* table, const char* column,
                              const int64_t* offsets, const char* chars, int64_t n,
                              const int8_t* nulls);
/* Enum dictionary: key k's string is chars[offsets[k] .. offsets[k+1]). */
int kdbo_register_enum(kdbo_ctx* ctx, int32_t enum_id, const int64_t* offsets,
                       const char* chars, int32_t n);

/* Skinner options: episode budget and UCT seed
 * (runtime/skinner_join_executor.cc:20-22). */
void kdbo_set_skinner_options(kdbo_ctx* ctx, int32_t budget_per_episode, int32_t seed);

int kdbo_execute(kdbo_ctx* ctx, const char* plan_json, kdbo_result** out);
/* Execution time of the last kdbo_execute in seconds (execute only). */
double kdbo_last_exec_seconds(kdbo_ctx* ctx);

int64_t kdbo_result_num_rows(const kdbo_result* r);
int32_t kdbo_result_num_cols(const kdbo_result* r);
/* writes "TYPE" or "ENUM:<id>" */
int kdbo_result_col_type(const kdbo_result* r, int32_t col, char* buf, int32_t cap);
int kdbo_result_get_i64(const kdbo_result* r, int32_t col, int64_t* out);
int kdbo_result_get_f64(const kdbo_result* r, int32_t col, double* out);
int kdbo_result_get_nulls(const kdbo_result* r, int32_t col, int8_t* out);
/* TEXT value at (col,row): returns length, copies up to cap bytes. */
int64_t kdbo_result_get_text(const kdbo_result* r, int32_t col, int64_t row, char* buf,
                             int64_t cap);
/* Whole result in the reference printer format; returns needed size + 1. */
int64_t kdbo_result_format(kdbo_ctx* ctx, const kdbo_result* r, char* buf, int64_t cap);
void kdbo_result_free(kdbo_result* r);

#ifdef __cplusplus
}
#endif

#endif /* KDB_ORACLE_H_ */
