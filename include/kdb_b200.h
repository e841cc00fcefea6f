/* kdb_b200.h -- C ABI of the B200 execution backend for KushDB's relational
 * hot path (ScanSelect -> HashJoin -> GroupByAggregate -> OrderBy, plus
 * SkinnerJoin).
 *
 * The reference calls its runtime per tuple from JIT-generated code through
 * raw function pointers (DeclareExternalFunction in compile/proxy).  Per-
 * tuple calls cannot cross to a GPU, so this boundary sits one level higher,
 * at operator-tree / operator-batch granularity:
 *
 *   reference                                        here
 *   -----------------------------------------------  --------------------------
 *   runtime::ColumnData::{Open,Size,Get}              kdb_table_add_column,
 *     (runtime/column_data.h:60-92),                  kdb_table_add_text_column,
 *     FileManager::Open (runtime/file_manager.cc:22)  kdb_column_open_kdb
 *   runtime::Enum::EnumManager::Register/GetKey       kdb_enum_register,
 *     (runtime/enum.h:17-40)                          kdb_enum_open_kdbenum
 *   compile::TranslateQuery + ExecutableQuery::      kdb_query_execute
 *     Execute (compile/query_translator.h:12,
 *     execution/executable_query.cc:199-255)
 *   runtime::HashTable::{Create,Insert,GetBucket}    device join tables built and
 *     (runtime/hash_table.h:22-38)                    probed inside the pipelines
 *                                                     of a HASH_JOIN plan
 *   runtime::AggregateHashTable::* + aggregators     device group tables of a
 *     (runtime/aggregate_hash_table.h:28-49,          GROUP_BY_AGGREGATE plan
 *      compile/proxy/aggregator.cc)
 *   runtime::Vector::Sort (runtime/vector.cc:105)    device sort of an ORDER_BY
 *                                                     plan
 *   runtime::ExecutePermutableSkinnerJoin            SKINNER_JOIN plan
 *     (runtime/skinner_join_executor.h:16-25)
 *   runtime::Printer (runtime/printer.cc)            kdb_result_format
 *
 * Conventions: every function returns 0 on success and a negative code on
 * error (no exceptions cross the ABI); kdb_last_error() describes the last
 * failure on a context.  Objects are opaque handles owned by a kdb_ctx (one
 * CUDA device, one stream).  A context is used by one host thread at a time.
 * Plans are passed as JSON text in the plan::Operator shape (see
 * kushdb_b200/plan.py for the serialiser).
 */
#ifndef KDB_B200_H_
#define KDB_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KDB_OK 0
#define KDB_ERR_INVALID -1      /* bad argument / plan */
#define KDB_ERR_CUDA -2         /* CUDA runtime / driver error */
#define KDB_ERR_COMPILE -3      /* NVRTC compilation failed */
#define KDB_ERR_CAPACITY -4     /* a device table or buffer ran out of room */
#define KDB_ERR_UNSUPPORTED -5  /* plan feature not supported */
#define KDB_ERR_TIMEOUT -6      /* a bounded device wait gave up */

typedef struct kdb_ctx kdb_ctx;
typedef struct kdb_result kdb_result;

/* ---- context ------------------------------------------------------------ */
/* Creates a context on CUDA device `device`.  Replaces QueryState/
 * FileManager ownership (execution/query_state.h:15-37). */
int kdb_ctx_create(int device, kdb_ctx** out);
int kdb_ctx_destroy(kdb_ctx* ctx);
const char* kdb_last_error(kdb_ctx* ctx);
/* Number of kernels this context launched since creation (all kinds). */
int64_t kdb_ctx_kernel_launches(kdb_ctx* ctx);
/* Bytes of device memory the context currently holds for columns. */
int64_t kdb_ctx_column_bytes(kdb_ctx* ctx);
/* The cudaStream_t all of the context's work is issued on (for callers that
 * time or order work around it with their own CUDA events). */
void* kdb_ctx_stream(kdb_ctx* ctx);
/* When enabled, every kernel launch of a query is bracketed by CUDA events;
 * kdb_last_query_kernels then reports them. */
int kdb_ctx_set_profiling(kdb_ctx* ctx, int enabled);
/* Per-kernel device times of the last query as JSON
 * [{"tag":"...","ms":x},...]; returns the size needed including the NUL. */
int64_t kdb_last_query_kernels(kdb_ctx* ctx, char* buf, int64_t cap);

/* ---- columns (runtime/column_data.h:20-92) -------------------------------
 * Type strings: "SMALLINT" "INT" "BIGINT" "REAL" "DATE" "TEXT" "BOOLEAN"
 * "ENUM:<id>".  Fixed-width data uses the type's physical width (int8
 * BOOLEAN, int16 SMALLINT, int32 INT/DATE/ENUM, int64 BIGINT, f64 REAL);
 * `nulls` (optional) holds one int8 per row, 1 = NULL (the reference's
 * `_null.kdb` BOOLEAN column).  Data is copied into HBM and stays resident
 * until the table is dropped or the context destroyed. */
int kdb_table_add_column(kdb_ctx* ctx, const char* table, const char* column, const char* type,
                         const void* host_data, int64_t n, const int8_t* host_nulls);
/* TEXT: value r is chars[offsets[r] .. offsets[r+1]) (offsets: n+1 int64). */
int kdb_table_add_text_column(kdb_ctx* ctx, const char* table, const char* column,
                              const int64_t* offsets, const char* chars, int64_t n,
                              const int8_t* host_nulls);
/* Reads a reference .kdb column file (runtime/column_data.cc:121-229 layout)
 * and, when `null_path` is non-empty, its BOOLEAN null file. */
int kdb_column_open_kdb(kdb_ctx* ctx, const char* table, const char* column, const char* type,
                        const char* path, const char* null_path);
int kdb_table_drop(kdb_ctx* ctx, const char* table);
int64_t kdb_table_num_rows(kdb_ctx* ctx, const char* table);

/* ---- enums (runtime/enum.cc) --------------------------------------------- */
/* Key k's string is chars[offsets[k] .. offsets[k+1]). */
int kdb_enum_register(kdb_ctx* ctx, int32_t enum_id, const int64_t* offsets, const char* chars,
                      int32_t n);
/* Reads a reference .kdbenum dictionary (runtime/enum.cc:38-131). */
int kdb_enum_open_kdbenum(kdb_ctx* ctx, int32_t enum_id, const char* path);

/* ---- queries -------------------------------------------------------------- */
/* Translates the plan into device pipelines (compiled for sm_100a through
 * NVRTC and cached by plan shape) and runs them; the result stays on the
 * host in `out`. */
int kdb_query_execute(kdb_ctx* ctx, const char* plan_json, kdb_result** out);
/* End to end from host memory: brings the listed fixed-width columns into
 * HBM (added, or refreshed in place when the table already holds a column of
 * that name, type and row count) and runs the plan over them, returning
 * when the result is on the host.  The copies are split into chunks spread
 * over several copy streams, all in flight together with no
 * synchronisation between columns (kdb_ctx_set_ingest); pinned host memory
 * copies at the full host-link rate.  Like kdb_table_add_column this changes
 * the tables, so prepared recordings of plans over them are dropped. */
typedef struct {
  const char* table;
  const char* column;
  const char* type;     /* as kdb_table_add_column */
  const void* data;     /* n values in the type's physical width */
  int64_t n;
  const int8_t* nulls;  /* optional, one byte per row, 1 = NULL */
} kdb_host_column;
int kdb_query_execute_host(kdb_ctx* ctx, const char* plan_json, const kdb_host_column* cols, int32_t ncols,
                           kdb_result** out);
/* Chunk size (>= 64 KiB) and copy streams (1-8) of host-to-device column
 * copies (kdb_query_execute_host); defaults 64 MiB and 2. */
int kdb_ctx_set_ingest(kdb_ctx* ctx, int64_t chunk_bytes, int32_t streams);
/* Device time (ms, CUDA events) of the last kdb_query_execute's pipelines,
 * excluding result download, and the bytes read from table columns. */
double kdb_last_query_device_ms(kdb_ctx* ctx);

/* Prepared queries (on by default): the first run of a plan text records
 * its launches; later runs of the same text over unchanged tables replay
 * them as one CUDA graph (no code generation or per-kernel launches) and
 * keep that plan's device buffers between runs.  Any table or enum change
 * invalidates them; Skinner joins and profiling runs are never replayed. */
int kdb_ctx_set_prepared_queries(kdb_ctx* ctx, int32_t on);

/* Code-generation switches and tuning values of the context, named KDB_*
 * (e.g. "KDB_NO_VECTOR_SCAN", "KDB_DENSE_BLOCK" = "128"): every measured
 * choice of the generated pipelines can be turned off or retuned through
 * one, for A/B comparisons.  A context starts from the KDB_* environment
 * variables present when it is created; value NULL removes an option.
 * Changing an option drops the prepared recordings.  kdb_ctx_get_option
 * returns 0 when the option is unset, else the size of its value with the
 * NUL (copied into buf when it fits cap). */
int kdb_ctx_set_option(kdb_ctx* ctx, const char* name, const char* value);
int64_t kdb_ctx_get_option(kdb_ctx* ctx, const char* name, char* buf, int64_t cap);

/* ---- Skinner join options (runtime/skinner_join_executor.cc:20-22) ------
 * Work budget per episode (tuples examined, the reference's
 * --budget_per_episode) and the UCT random seed (--join_seed).  Join order
 * changes only the emission order, never the result set. */
int kdb_ctx_set_skinner(kdb_ctx* ctx, int64_t budget_per_episode, uint32_t seed);
/* Episodes the last SKINNER_JOIN of the last query ran. */
int64_t kdb_last_skinner_episodes(kdb_ctx* ctx);
/* Tuples examined by all episodes of the last Skinner join. */
int64_t kdb_last_skinner_work(kdb_ctx* ctx);
/* Episode batches of the last Skinner join.  The episodes run in batches
 * (option KDB_SKINNER_BATCH, 1-16, default 8): the search picks the next
 * join orders before the running ones report their rewards (the statistics
 * are corrected when they do), and a batch shares one set of launches and
 * one read-back.  Each episode's slice and offsets are those a one-at-a-
 * time run would give it, so results stay exactly-once. */
int64_t kdb_last_skinner_batches(kdb_ctx* ctx);

/* ---- learned join-order prior (no reference counterpart) ----------------
 * A 64 -> 128 -> 128 -> 128 -> 1 ReLU MLP (fp32) predicting the episode
 * reward of appending a table to a join-order prefix, with hand-written
 * CUDA forward / backward / Adam kernels.  Policies of the Skinner join:
 *   0 UCT as the reference (runtime/skinner_join_executor.cc:779-838);
 *   1 UCT seeded by the prior: every action starts as tried once with the
 *     predicted reward and playouts follow the prior, observed rewards
 *     overrule it; joins of more than 8 tables fall back to 0;
 *   2 uniformly random connected orders (collects training data).
 * The policy never changes a result, only the order search.  With
 * log_samples set, every (prefix, next table) step of every episode is
 * recorded as a feature row and the episode's reward. */
typedef struct kdb_mlp kdb_mlp;
int32_t kdb_mlp_num_features(void);
int64_t kdb_mlp_num_params(void);
int kdb_mlp_create(kdb_ctx* ctx, uint32_t seed, kdb_mlp** out);
const char* kdb_mlp_last_error(kdb_mlp* m);
int kdb_mlp_set_params(kdb_mlp* m, const float* params, int64_t n);
int kdb_mlp_get_params(kdb_mlp* m, float* params, int64_t n);
/* n <= 4096 rows of kdb_mlp_num_features() floats -> n predictions */
int kdb_mlp_forward(kdb_mlp* m, const float* x, int64_t n, float* y);
/* gradient of mean((y - t)^2) w.r.t. every parameter, without an update */
int kdb_mlp_gradient(kdb_mlp* m, const float* x, const float* t, int64_t n, float* grad, double* loss);
/* one Adam step (beta 0.9 / 0.999); loss before the step */
int kdb_mlp_train_step(kdb_mlp* m, const float* x, const float* t, int64_t n, float lr, double* loss);
void kdb_mlp_free(kdb_mlp* m);
/* The model must outlive its use by the context. */
int kdb_ctx_set_skinner_policy(kdb_ctx* ctx, int32_t policy, kdb_mlp* prior, int32_t log_samples);
/* Samples of the last Skinner join with logging on: copies min(n, cap) rows
 * of features (row-major) and rewards; returns n. */
int64_t kdb_last_skinner_samples(kdb_ctx* ctx, float* features, float* rewards, int64_t cap);

/* ---- device sort (runtime/vector.cc:45-110) ------------------------------
 * Stable sort of n (key, value) pairs already in device memory by the low
 * `key_bits` bits of the keys (ties keep their input order); the primitive
 * under ORDER BY.  Scratch comes from the context's stream-ordered pool; the
 * call returns when the sort is done. */
int kdb_sort_pairs(kdb_ctx* ctx, uint64_t* d_keys, uint32_t* d_vals, int64_t n, int32_t key_bits);

/* The same sort without any device allocation, for callers that cannot
 * allocate when they sort: code running inside a CUDA host callback or
 * another context where CUDA allocation calls are not allowed, and host
 * engines that hand out every byte of HBM through their own allocator and
 * forbid a library's hidden allocations.  This entry point has no
 * counterpart in the reference.
 *
 * Scratch is one static device array sized for KDB_SORT_NOALLOC_MAX_PAIRS
 * pairs (12.25 MiB), held by every GPU that loads this library until the
 * process exits.  n above that limit returns KDB_ERR_CAPACITY without
 * launching anything.  The work is queued on `stream` (a cudaStream_t; NULL =
 * legacy default stream) on the current device and the call returns without
 * waiting.  The first call on each device looks up the array's device address
 * once (cudaGetSymbolAddress): make that first call before any stream
 * capture; resetting the device (cudaDeviceReset) after that first call is
 * not supported, because the looked-up address is kept.  An error already
 * pending on the calling thread (cudaPeekAtLastError) is left in place and
 * the call returns KDB_ERR_CUDA without launching.  Every call shares the one
 * array, so calls whose work overlaps on the GPU (different streams, or
 * different host threads) race and must be ordered by the caller. */
#define KDB_SORT_NOALLOC_MAX_PAIRS (1 << 20)
int kdb_sort_pairs_noalloc(uint64_t* d_keys, uint32_t* d_vals, int64_t n, int32_t key_bits,
                           void* stream);

/* ---- per-operator boundary ------------------------------------------------
 * One operator per call over HBM-resident tables, for hosts that drive the
 * operators themselves the way the reference's generated code calls one
 * runtime structure at a time.  Objects belong to the context that made them
 * and must be freed before it is destroyed.
 *
 * Selection vectors: ascending row ids of one table.  kdb_scan_select
 * replaces ScanSelectTranslator::Produce (compile/translators/
 * scan_select_translator.cc:92-156): `filter_json` is one BOOLEAN expression
 * in the plan JSON shape over `columns` (bound by position: VIRTUAL_COLUMN_REF
 * or COLUMN_REF of child 0 with column_idx = position), with the reference's
 * three-valued logic; a row qualifies when the filter is TRUE. */
typedef struct kdb_selvec kdb_selvec;
int kdb_scan_select(kdb_ctx* ctx, const char* table, const char* const* columns, int32_t ncols,
                    const char* filter_json, kdb_selvec** out);
int64_t kdb_selvec_size(const kdb_selvec* s);
/* copies min(cap, size) row ids to host memory; returns the size */
int64_t kdb_selvec_get(const kdb_selvec* s, int32_t* rows, int64_t cap);
/* device array of the row ids (valid until the vector is freed) */
const int32_t* kdb_selvec_device_rows(const kdb_selvec* s);
void kdb_selvec_free(kdb_selvec* s);

/* Sort of a table's rows: the rows of `table` (all, or those of `sel`) in
 * ORDER BY order of nkeys key columns, asc[k] != 0 ascending, as a selection
 * vector in that order (not ascending).  Replaces OrderByTranslator
 * (compile/translators/order_by_translator.cc:35-110) over runtime::Vector's
 * merge sort (runtime/vector.cc:45-110): a NULL key sorts after every value
 * ascending and before every value descending (proxy::LessThan used both
 * ways), ENUM keys in string order, and rows whose keys tie keep their input
 * order.  Keys: SMALLINT/INT/BIGINT/DATE/BOOLEAN/ENUM/REAL columns (TEXT:
 * KDB_ERR_UNSUPPORTED). */
int kdb_sort(kdb_ctx* ctx, const char* table, const char* const* key_columns, const int8_t* asc, int32_t nkeys,
             const kdb_selvec* sel, kdb_selvec** out);

/* Hash join build / probe: runtime::HashTable::{Create,Insert,GetBucket}
 * (runtime/hash_table.h:22-38) as hash_join_translator.cc:79-139 drives it.
 * The key is one SMALLINT/INT/BIGINT/DATE/ENUM/BOOLEAN column; rows with a
 * NULL key are not inserted (and never match), duplicates are all kept.
 * sel NULL = every row.  load_factor in (0.05, 0.95].  fanout: 1 = one
 * open-addressing table; a power of two up to 8192 = that many sub-tables
 * chosen by the key hash's top bits (radix partitioned: both sides are
 * scattered by partition and each partition joins in shared memory, its
 * sub-table and probe tiles brought in by TMA bulk copies); 0 = one table
 * while it fits well inside L2, partitioned above. */
typedef struct kdb_hash kdb_hash;
typedef struct kdb_pairs kdb_pairs;
int kdb_hash_build(kdb_ctx* ctx, const char* table, const char* key_column, const kdb_selvec* sel,
                   double load_factor, int32_t fanout, kdb_hash** out);
int kdb_hash_info(const kdb_hash* h, int32_t* fanout, int64_t* slots, int64_t* bytes);
/* Every (probe row, build row) pair with equal keys.  ordered != 0: sorted
 * by probe row, then build row -- the reference's order, in which a probe
 * row meets its bucket's rows in insertion order; 0: in no particular order.
 * The probe key must have the build key's width class (BIGINT with BIGINT,
 * the narrower types among themselves). */
int kdb_hash_probe(kdb_ctx* ctx, const kdb_hash* h, const char* table, const char* key_column,
                   const kdb_selvec* sel, int32_t ordered, kdb_pairs** out);
void kdb_hash_free(kdb_hash* h);
int64_t kdb_pairs_size(const kdb_pairs* p);
int64_t kdb_pairs_get(const kdb_pairs* p, int32_t* probe_rows, int32_t* build_rows, int64_t cap);
void kdb_pairs_free(kdb_pairs* p);

/* Group-by aggregation: runtime::AggregateHashTable with the proxy
 * aggregators (runtime/aggregate_hash_table.h:28-49, compile/proxy/
 * aggregate_hash_table.cc:187-333, compile/proxy/aggregator.cc:28-296).
 * 1-4 integer/date/enum/boolean key columns (NULL is a key value of its
 * own) and 1-8 aggregates over numeric columns of the same table:
 * SUM/MIN/MAX keep the input type (integer sums wrap at its width), AVG is
 * REAL, COUNT is BIGINT (column NULL = rows; COUNT(col) counts the non-NULL
 * values plus the group's first row when that one is NULL, as the reference
 * does); a SUM/MIN/MAX/AVG of only NULLs is NULL.  max_groups bounds the
 * groups (<= 0: the table's row count); more return KDB_ERR_CAPACITY and the
 * table is then unusable.  Updates accumulate (one per morsel/selection);
 * the result lists the groups in first-insertion order, keys first, then
 * the aggregates.  Float sums differ from sequential ones only in summation
 * order.  Pre-aggregation in shared memory is on by default. */
#define KDB_AGG_SUM 0
#define KDB_AGG_MIN 1
#define KDB_AGG_MAX 2
#define KDB_AGG_AVG 3
#define KDB_AGG_COUNT 4
typedef struct {
  int32_t agg;
  const char* column;
} kdb_agg_spec;
typedef struct kdb_agg kdb_agg;
int kdb_agg_create(kdb_ctx* ctx, const char* table, const char* const* key_columns, int32_t nkeys,
                   const kdb_agg_spec* aggs, int32_t naggs, int64_t max_groups, kdb_agg** out);
int kdb_agg_set_pre_aggregation(kdb_agg* a, int32_t on);
int kdb_agg_update(kdb_ctx* ctx, kdb_agg* a, const kdb_selvec* sel);
int kdb_agg_finalize(kdb_ctx* ctx, kdb_agg* a, kdb_result** out);
void kdb_agg_free(kdb_agg* a);

/* Column indexes: key -> ascending row ids.  kdb_index_build replaces
 * runtime::MemoryColumnIndex (runtime/memory_column_index.cc:17-121) over a
 * resident column; kdb_index_open_kdbindex reads a reference .kdbindex file
 * (runtime/column_index.h:21-41, runtime/column_index.cc:67-144; integer,
 * date, enum and boolean keys).  NULL keys are not indexed. */
typedef struct kdb_index kdb_index;
int kdb_index_build(kdb_ctx* ctx, const char* table, const char* column, kdb_index** out);
int kdb_index_open_kdbindex(kdb_ctx* ctx, const char* path, const char* type, kdb_index** out);
int64_t kdb_index_num_keys(const kdb_index* i);
int64_t kdb_index_num_rows(const kdb_index* i);
/* distinct keys in ascending order (copies min(cap, n)); returns n */
int64_t kdb_index_keys(const kdb_index* i, int64_t* keys, int64_t cap);
/* rows of `key` (copies min(cap, n)); returns n (0 for an absent key) */
int64_t kdb_index_get(const kdb_index* i, int64_t key, int32_t* rows, int64_t cap);
void kdb_index_free(kdb_index* i);

/* The Skinner join operator on its own: runtime::ExecutePermutableSkinnerJoin
 * (runtime/skinner_join_executor.h:16-25).  skinner_json is one SKINNER_JOIN
 * operator in the plan JSON shape whose children are scans; policy as in
 * kdb_ctx_set_skinner_policy (0 UCT, 1 learned prior, 2 random), the budget
 * and seed as in kdb_ctx_set_skinner, for this call only.  The result rows
 * are the operator's output schema. */
int kdb_skinner_execute(kdb_ctx* ctx, const char* skinner_json, int32_t policy, int64_t budget_per_episode,
                        uint32_t seed, kdb_result** out);

/* ---- batched form ----------------------------------------------------------
 * Many queries of one template, run together as a captured CUDA graph of
 * fused kernels (one launch per phase for all queries):
 *   SELECT d.key, SUM(f.price * (1 - f.disc)) FROM dim d JOIN fact f
 *   ON f.fk = d.key WHERE d.date < date_lt AND d.seg = seg GROUP BY d.key
 * i.e. HashJoin(ScanSelect(dim), Scan(fact)) -> GroupByAggregate
 * (hash_join_translator.cc:34-139, group_by_aggregate_translator.cc:36-111)
 * with per-query constants.  The dimension key must be unique (a primary
 * key); kdb_batch_run reports KDB_ERR_UNSUPPORTED otherwise.  Columns are
 * registered tables' columns (int32 key/date/seg/fk, REAL price/disc). */
typedef struct kdb_batch kdb_batch;
typedef struct {
  const char* dim_table;
  const char* dim_key;
  const char* dim_date;
  const char* dim_seg;
  const char* fact_table;
  const char* fact_fk;
  const char* fact_price;
  const char* fact_disc;
  int32_t date_lt;
  int32_t seg;
} kdb_batch_query;
int kdb_batch_create(kdb_ctx* ctx, const kdb_batch_query* queries, int32_t n, kdb_batch** out);
/* block in {128,256,512}, load factor of the join tables in (0.05, 0.95],
 * fanout = power-of-two number of join sub-tables per query (radix
 * partitioning by the key hash's top bits). */
int kdb_batch_configure(kdb_batch* b, int32_t block, double load_factor, int32_t fanout);
/* Autotuner: times every block x load factor {0.5,0.7,0.9} x fanout
 * {1,64,256,1024} configuration (`reps` replays each), keeps the fastest;
 * writes a JSON report of all timings into `report`. */
int kdb_batch_tune(kdb_batch* b, int32_t reps, char* report, int64_t cap);
int kdb_batch_config(kdb_batch* b, int32_t* block, double* load_factor, int32_t* fanout);
/* Runs all queries (graph replay) and waits. */
int kdb_batch_run(kdb_batch* b);
/* Mean device ms per batch over `reps` replays (CUDA events), -1 on error. */
double kdb_batch_run_timed(kdb_batch* b, int32_t reps);
/* Query q's groups (key, sum) in the order the fact stream first reaches
 * them; returns the group count (copies at most `cap`). */
int64_t kdb_batch_result(kdb_batch* b, int32_t q, int32_t* keys, double* sums, int64_t cap);
void kdb_batch_free(kdb_batch* b);

/* ---- serving ---------------------------------------------------------------
 * A request loop over the context's resident tables (no reference
 * counterpart: the reference runs one query per process,
 * execution/executable_query.cc:199-255).  `slots` worker threads, each with
 * its own CUDA stream, take queued plans as soon as a slot is free and the
 * request's estimated device footprint fits `hbm_budget_bytes` beside the
 * ones in flight, so queries of different shapes run concurrently.  Tables
 * must not be added or dropped while a server runs.  A quarter of the budget
 * holds build state kept across requests: the filtered children of Skinner
 * joins and their join-column indexes, reused by later requests that read
 * the same children (requests are admitted against the other three
 * quarters). */
typedef struct kdb_server kdb_server;
int kdb_server_start(kdb_ctx* ctx, int32_t slots, int64_t hbm_budget_bytes, kdb_server** out);
/* Queues a plan (same JSON as kdb_query_execute); returns a ticket > 0 or a
 * negative KDB_ERR_* (a plan that does not parse is rejected here). */
int64_t kdb_server_submit(kdb_server* s, const char* plan_json);
/* 1 = still pending, 0 = done (the result is handed over in *out and the
 * ticket retired), < 0 = the query failed (message in kdb_last_error of the
 * owning context).  Waits up to wait_ms for completion. */
int kdb_server_poll(kdb_server* s, int64_t ticket, int64_t wait_ms, kdb_result** out);
/* JSON: completed, failed, p50_ms, p99_ms, max_ms (submission to completion),
 * service_p50_ms, queries_per_second, peak_in_flight, slots, hbm_budget (the
 * admission budget), kernel_launches, build_cache_hits, build_cache_misses,
 * build_cache_bytes, build_cache_entries.
 * Returns the size needed including the NUL. */
int64_t kdb_server_stats(kdb_server* s, char* buf, int64_t cap);
/* Finishes the requests in flight, drops queued ones, joins the workers. */
void kdb_server_stop(kdb_server* s);

/* ---- results (runtime/printer.cc output format) ------------------------ */
int64_t kdb_result_num_rows(const kdb_result* r);
int32_t kdb_result_num_cols(const kdb_result* r);
int kdb_result_col_type(const kdb_result* r, int32_t col, char* buf, int32_t cap);
int kdb_result_get_i64(const kdb_result* r, int32_t col, int64_t* out);
int kdb_result_get_f64(const kdb_result* r, int32_t col, double* out);
int kdb_result_get_nulls(const kdb_result* r, int32_t col, int8_t* out);
int64_t kdb_result_get_text(const kdb_result* r, int32_t col, int64_t row, char* buf, int64_t cap);
/* Whole result in the reference printer format ("v|v|...|\n" per row);
 * returns the size needed including the terminating NUL. */
int64_t kdb_result_format(kdb_ctx* ctx, const kdb_result* r, char* buf, int64_t cap);
void kdb_result_free(kdb_result* r);

#ifdef __cplusplus
}
#endif

#endif /* KDB_B200_H_ */
