/*
 * shwfs_bin.h -- the MAOS .bin array file format (read and write).
 *
 * The format of sys/bin.c and math/cell.c, math/spbin.c of the reference,
 * byte for byte: each array is an optional header string (M_COMMENT, its
 * length rounded up to 8 bytes, the text, the length again, M_COMMENT), the
 * padding magic M_SKIP, then the type magic and the two uint64 dimensions
 * (write_bin_header, sys/bin.c:762-790), then the data in column-major order.
 * A cell (MCC_ANY) is followed by its nx*ny members, an empty member written
 * as a header of the first non-empty member's type with zero size
 * (writedata, math/cell.c:300-328).  A sparse matrix holds after its header
 * the uint64 number of non-zeros, the column pointers (ny+1), the row indices
 * and the values (spwritedata, math/spbin.c:26-43).  Files whose name ends in
 * ".gz" are gzip streams; reading accepts either form whatever the name.
 * Integers are little-endian as on the machines the reference writes on.
 */
#ifndef SHWFS_BIN_H
#define SHWFS_BIN_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Type magics of sys/bin.h:51-81 (the values may not change). */
#define SHWFS_M_DBL 0x6402u
#define SHWFS_M_INT64 0x6403u
#define SHWFS_M_CMP 0x6404u
#define SHWFS_M_INT32 0x6405u
#define SHWFS_M_FLT 0x6408u
#define SHWFS_M_ZMP 0x6409u
#define SHWFS_M_INT8 0x640Au
#define SHWFS_M_INT16 0x640Bu
#define SHWFS_MCC_ANY 0x6421u
#define SHWFS_M_CSP64 0x6400u
#define SHWFS_M_DSP64 0x6401u
#define SHWFS_M_CSP32 0x6406u
#define SHWFS_M_DSP32 0x6407u
#define SHWFS_M_SSP64 0x6430u
#define SHWFS_M_SSP32 0x6431u
#define SHWFS_M_ZSP64 0x6432u
#define SHWFS_M_ZSP32 0x6433u
#define SHWFS_M_COMMENT 0x6500u
#define SHWFS_M_SKIP 0x6600u
#define SHWFS_M_EOD 0x64FFu

/* One array of a .bin file.  Dense (id & 0xFFFF of a dense type, which also
   covers map_t/loc_t ids such as 0x016402): data holds nx*ny elements.
   Sparse: nnz, pp (ny+1), pi (nnz) as int64 whatever the file's index width,
   data the nnz values; an empty sparse matrix has nx = ny = 0.  Cell
   (SHWFS_MCC_ANY): cells holds nx*ny members, NULL for an empty one. */
typedef struct shwfs_bin {
	uint32_t id;
	uint64_t nx, ny;
	char* keywords;          /* header text or NULL */
	void* data;
	uint64_t nnz;            /* sparse only */
	int64_t *pp, *pi;        /* sparse only */
	struct shwfs_bin** cells;  /* cell only */
} shwfs_bin;

/* Bytes per element of a dense or sparse-value type, 0 for others. */
int shwfs_bin_elsize(uint32_t id);
/* 1 for the sparse types. */
int shwfs_bin_is_sparse(uint32_t id);

/* New arrays (data copied; keywords may be NULL).  A cell's members are
   set through ->cells and owned by the cell. */
shwfs_bin* shwfs_bin_new_dense(uint32_t id, uint64_t nx, uint64_t ny, const void* data, const char* keywords);
shwfs_bin* shwfs_bin_new_sparse(uint32_t id, uint64_t nx, uint64_t ny, uint64_t nnz, const int64_t* pp,
	const int64_t* pi, const void* px, const char* keywords);
shwfs_bin* shwfs_bin_new_cell(uint64_t nx, uint64_t ny, const char* keywords);
void shwfs_bin_free(shwfs_bin* a);

/* Reads the first array of a file (readbin, math/cell.c:545-559, without the
   scan of several top-level arrays, which shwfs_bin_read_all gives).
   Returns 0 and *out (NULL for an empty file), or a negative error. */
int shwfs_bin_read(const char* path, shwfs_bin** out);
/* Reads every top-level array of a file into a cell of n x 1 (zfarr dumps
   and files holding several arrays one after another). */
int shwfs_bin_read_all(const char* path, shwfs_bin** out);
/* Writes an array (writebin, math/cell.c:330-337); a NULL array writes an
   empty cell.  Returns 0 or a negative error. */
int shwfs_bin_write(const char* path, const shwfs_bin* a);
/* Message of the last error of this thread. */
const char* shwfs_bin_error(void);

#define SHWFS_BIN_EIO (-1)     /* open, read or write failed */
#define SHWFS_BIN_EFORMAT (-2) /* not a valid .bin stream */
#define SHWFS_BIN_ENOMEM (-3)
#define SHWFS_BIN_EINVAL (-4)

#ifdef __cplusplus
}
#endif
#endif
