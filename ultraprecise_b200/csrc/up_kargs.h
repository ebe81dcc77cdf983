// up_kargs.h — the argument blocks of the generated kernels, declared once.
//
// The host launch code includes this header (through up_internal.h) to fill
// the blocks, and every NVRTC-compiled kernel includes it (through
// up_dev.cuh, which the JIT registers together with this header), so a
// kernel and its launcher can never disagree on a field's position.  Plain C
// layout with fixed-width members only (64-bit pointers and integers on both
// sides); the static_asserts pin the sizes the generated code was written for.
#ifndef UP_KARGS_H_
#define UP_KARGS_H_

#define UP_MAX_COLS 16
#define UP_MAX_AGGS 16
#define UP_BATCH_MAX_COLS 8

// One kernel input column: the reference's AriesColumnDataIterator shape
// (contiguous data, or a block list with row prefix sums, and an optional
// int32 row indirection where -1 is NULL).
struct UpKCol {
    const unsigned char* data;
    const unsigned char* const* blocks;
    const long long* prefix;
    const int* indices;
    int n_blocks;
    int value_bytes;
};

// Expression modules (up_expr_tile / up_expr_generic).
struct UpArgs {
    UpKCol col[UP_MAX_COLS];
    long long rows;
    unsigned char* out;
    unsigned int* err;
    int vec_ok;
    int out_nullable;
};

// Query modules (up_query_*).  key_mode 0: group ids from gid[]; otherwise
// the group is key_table[key] with key = key0[r] (1), key0[r] << 8 | key1[r]
// (2), or key0[2r] << 8 | key0[2r+1] (3).  n_groups < 0: the count is read
// from the key table on the device, -n_groups being the capacity.
struct UpQArgs {
    UpKCol col[UP_MAX_COLS];
    unsigned char* out[UP_MAX_AGGS];
    long long rows;
    const int* gid;
    unsigned int* acc;
    unsigned long long* cnt;
    unsigned int* err;
    int n_groups;
    int vec_ok;
    const unsigned char* key0;
    const unsigned char* key1;
    const int* key_table;
    int key_mode;
};

// Batch modules: one task of the work queue, and the band kernels' arguments.
struct BTask {
    UpKCol col[UP_BATCH_MAX_COLS];
    long long rows;
    unsigned char* out;
    const int* gid;
    unsigned int* acc;
    unsigned long long* cnt;
    int n_groups;
    int words;
};
struct BArgs {
    BTask* tasks;
    const int* item_task;
    const long long* item_tile;
    long long n_items;
    unsigned long long* head;
    unsigned int* err;
    int tile_rows;
    int pad;
};

// Merged launches of one expression module (the serving loop): up_expr_multi
// walks virtual tiles of R rows over every request, request k owning tiles
// [tile0_k, tile0_{k+1}); each request has its own columns, output and error word.
struct UpMultiReq {
    UpKCol col[UP_MAX_COLS];
    long long rows;
    unsigned char* out;
    unsigned int* err;
    long long tile0;
    int vec_ok;
    int pad;
};
struct UpMultiArgs {
    const UpMultiReq* req;
    long long n_tiles;
    int n_req;
    int pad;
};

#if defined(__cplusplus) && __cplusplus >= 201103L
static_assert(sizeof(UpMultiReq) == 680, "UpMultiReq layout");
static_assert(sizeof(UpMultiArgs) == 24, "UpMultiArgs layout");
static_assert(sizeof(UpKCol) == 40, "UpKCol layout");
static_assert(sizeof(UpArgs) == 672, "UpArgs layout");
static_assert(sizeof(UpQArgs) == 848, "UpQArgs layout");
static_assert(sizeof(BTask) == 368, "BTask layout");
static_assert(sizeof(BArgs) == 56, "BArgs layout");
#endif

#endif  // UP_KARGS_H_
