/*
 * up_oracle.h — CPU oracle for the exact-decimal path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and its
 * reference arm) load it.  The product library never links or calls it.
 *
 * It restates UltraPrecise's decimal semantics in plain C; each function in
 * up_oracle.c cites the reference file:line it follows.  Parity pin: the
 * restatement is checked against golden vectors produced by the reference's
 * own AriesDecimal<LEN> device code (oracle/ref/, tests/golden/) and against
 * an independent Python-int restatement (oracle/pyref.py).
 */
#ifndef UP_ORACLE_H_
#define UP_ORACLE_H_

#include <stdint.h>
#include "../include/ultraprecise.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXL 400

typedef struct orc_dec {
    uint32_t sign;
    int32_t frac;
    int32_t n;                 /* significant limbs (m[n-1] != 0, or n == 0) */
    uint32_t m[ORC_MAXL];      /* little-endian base-2^32 magnitude */
} orc_dec;

int32_t orc_compact_bytes(int32_t precision);
int32_t orc_precision_words(int32_t precision);

void orc_decode(const uint8_t* bytes, int32_t nbytes, int32_t frac, orc_dec* out);
/* returns UP_ROWERR_OVERFLOW when magnitude bits were lost */
uint32_t orc_encode(const orc_dec* v, int32_t nbytes, uint8_t* out);

void orc_add(orc_dec* r, const orc_dec* a, const orc_dec* b);
void orc_sub(orc_dec* r, const orc_dec* a, const orc_dec* b);
void orc_mul(orc_dec* r, const orc_dec* a, const orc_dec* b);
uint32_t orc_div(orc_dec* r, const orc_dec* a, const orc_dec* b);
uint32_t orc_mod(orc_dec* r, const orc_dec* a, const orc_dec* b);
void orc_rescale(orc_dec* r, const orc_dec* a, int32_t scale);
/* op: UP_NODE_LT .. UP_NODE_NE */
int32_t orc_compare(int32_t op, const orc_dec* a, const orc_dec* b);

/* Evaluate a typed expression for rows [0, rows).  cols[k] is a contiguous
 * host column of col_types[k] values (compact bytes).  out has rows*out_bytes
 * bytes (1 byte per row for comparisons).  err (may be NULL) gets the OR of
 * per-row UP_ROWERR_* bits; row_err (may be NULL) gets per-row bits. */
int32_t orc_eval_expr(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                      const up_col_type* col_types, const uint8_t* const* cols,
                      int64_t row_begin, int64_t row_end,
                      uint8_t* out, int32_t out_bytes, uint32_t* err, uint8_t* row_err);

/* The same over `threads` host threads (rows split in contiguous chunks). */
int32_t orc_eval_expr_mt(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                         const up_col_type* col_types, const uint8_t* const* cols,
                         int64_t rows, uint8_t* out, int32_t out_bytes, uint32_t* err,
                         int32_t threads);

/* Grouped aggregation of one compact column: SUM/AVG -> 133-byte images,
 * COUNT -> int64 per group.  group_ids[i] in [0, n_groups). */
int32_t orc_group_agg(const uint8_t* vals, int32_t value_bytes, int32_t scale,
                      int32_t kind, const int32_t* group_ids, int64_t rows,
                      int32_t n_groups, uint8_t* out);

/* Fused query: per row evaluate each aggregate's expression and aggregate it
 * by group (SUM/AVG/COUNT), over `threads` host threads. */
int32_t orc_query(const up_expr_node* nodes, int32_t n_nodes,
                  const up_col_type* col_types, const uint8_t* const* cols,
                  const up_query_agg* aggs, int32_t n_aggs,
                  const int32_t* group_ids, int64_t rows, int32_t n_groups,
                  uint8_t* const* outs, int32_t threads);

/* AVG division of one 133-byte SUM image by a count (DivisionInt64). */
void orc_division_int64(const uint8_t* sum_img, int64_t count, uint8_t* out_img);

#ifdef __cplusplus
}
#endif
#endif
