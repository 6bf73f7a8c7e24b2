/*
 * The MAOS .bin array file format: reader and writer.  The byte layout is the
 * reference's (sys/bin.c:693-790 headers, sys/bin.c:1115-1150 dense arrays,
 * math/cell.c:300-328 and 398-452 cells, math/spbin.c:26-84 sparse
 * matrices); files written here are byte-identical to the reference's for the
 * same arrays and keywords.  zlib streams carry both plain and gzip files.
 */
#include "../../../include/shwfs_bin.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

static __thread char g_err[256];

static int err(int code, const char* msg, const char* path) {
	snprintf(g_err, sizeof(g_err), "%s%s%s", msg, path ? ": " : "", path ? path : "");
	return code;
}

const char* shwfs_bin_error(void) { return g_err; }

int shwfs_bin_elsize(uint32_t id) {
	switch (id & 0xFFFFu) {
	case SHWFS_M_DBL: case SHWFS_M_INT64: case SHWFS_M_ZMP: return 8;
	case SHWFS_M_CMP: return 16;
	case SHWFS_M_INT32: case SHWFS_M_FLT: return 4;
	case SHWFS_M_INT16: return 2;
	case SHWFS_M_INT8: return 1;
	case SHWFS_M_DSP64: case SHWFS_M_DSP32: return 8;
	case SHWFS_M_SSP64: case SHWFS_M_SSP32: return 4;
	case SHWFS_M_CSP64: case SHWFS_M_CSP32: return 16;
	case SHWFS_M_ZSP64: case SHWFS_M_ZSP32: return 8;
	default: return 0;
	}
}

int shwfs_bin_is_sparse(uint32_t id) {
	switch (id) {
	case SHWFS_M_DSP64: case SHWFS_M_DSP32: case SHWFS_M_SSP64: case SHWFS_M_SSP32:
	case SHWFS_M_CSP64: case SHWFS_M_CSP32: case SHWFS_M_ZSP64: case SHWFS_M_ZSP32: return 1;
	default: return 0;
	}
}

static int sparse_index64(uint32_t id) {
	return id == SHWFS_M_DSP64 || id == SHWFS_M_SSP64 || id == SHWFS_M_CSP64 || id == SHWFS_M_ZSP64;
}

/* ---------------------------------------------------------------- arrays */
static char* dupstr(const char* s) { return s ? strdup(s) : NULL; }

shwfs_bin* shwfs_bin_new_dense(uint32_t id, uint64_t nx, uint64_t ny, const void* data, const char* keywords) {
	const int es = shwfs_bin_elsize(id);
	if (!es || shwfs_bin_is_sparse(id) || id == SHWFS_MCC_ANY) return NULL;
	shwfs_bin* a = (shwfs_bin*)calloc(1, sizeof(shwfs_bin));
	if (!a) return NULL;
	a->id = id;
	a->nx = nx;
	a->ny = ny;
	a->keywords = dupstr(keywords);
	const uint64_t n = nx * ny * (uint64_t)es;
	if (n) {
		a->data = malloc(n);
		if (!a->data) {
			shwfs_bin_free(a);
			return NULL;
		}
		if (data) memcpy(a->data, data, n);
		else memset(a->data, 0, n);
	}
	return a;
}

shwfs_bin* shwfs_bin_new_sparse(uint32_t id, uint64_t nx, uint64_t ny, uint64_t nnz, const int64_t* pp,
	const int64_t* pi, const void* px, const char* keywords) {
	if (!shwfs_bin_is_sparse(id)) return NULL;
	shwfs_bin* a = (shwfs_bin*)calloc(1, sizeof(shwfs_bin));
	if (!a) return NULL;
	a->id = id;
	a->nx = nx;
	a->ny = ny;
	a->nnz = nnz;
	a->keywords = dupstr(keywords);
	const int es = shwfs_bin_elsize(id);
	a->pp = (int64_t*)calloc(ny + 1, sizeof(int64_t));
	a->pi = (int64_t*)malloc((nnz ? nnz : 1) * sizeof(int64_t));
	a->data = malloc((nnz ? nnz : 1) * (size_t)es);
	if (!a->pp || !a->pi || !a->data) {
		shwfs_bin_free(a);
		return NULL;
	}
	if (pp) memcpy(a->pp, pp, (ny + 1) * sizeof(int64_t));
	if (pi && nnz) memcpy(a->pi, pi, nnz * sizeof(int64_t));
	if (px && nnz) memcpy(a->data, px, nnz * (size_t)es);
	return a;
}

shwfs_bin* shwfs_bin_new_cell(uint64_t nx, uint64_t ny, const char* keywords) {
	shwfs_bin* a = (shwfs_bin*)calloc(1, sizeof(shwfs_bin));
	if (!a) return NULL;
	a->id = SHWFS_MCC_ANY;
	a->nx = nx;
	a->ny = ny;
	a->keywords = dupstr(keywords);
	if (nx && ny) {
		a->cells = (shwfs_bin**)calloc(nx * ny, sizeof(shwfs_bin*));
		if (!a->cells) {
			shwfs_bin_free(a);
			return NULL;
		}
	}
	return a;
}

void shwfs_bin_free(shwfs_bin* a) {
	if (!a) return;
	if (a->cells)
		for (uint64_t i = 0; i < a->nx * a->ny; i++) shwfs_bin_free(a->cells[i]);
	free(a->cells);
	free(a->keywords);
	free(a->data);
	free(a->pp);
	free(a->pi);
	free(a);
}

/* ---------------------------------------------------------------- reading */
typedef struct {
	gzFile gz;
	const char* path;
} reader;

/* Reads exactly n bytes: 0 on success, 1 at a clean end of file (nothing
   read), negative on a short read or an error. */
static int rd(reader* r, void* buf, uint64_t n) {
	char* p = (char*)buf;
	uint64_t got = 0;
	while (got < n) {
		const uint64_t want = n - got > (1u << 30) ? (1u << 30) : n - got;
		const int k = gzread(r->gz, p + got, (unsigned)want);
		if (k < 0) return err(SHWFS_BIN_EIO, "read failed", r->path);
		if (k == 0) return got == 0 ? 1 : err(SHWFS_BIN_EFORMAT, "truncated file", r->path);
		got += (uint64_t)k;
	}
	return 0;
}

typedef struct {
	uint32_t id;
	uint64_t nx, ny;
	char* str;
} header;

/* read_bin_header (sys/bin.c:693-745): header strings are concatenated,
   padding magics skipped.  0: header read; 1: end of data; < 0: error. */
static int read_header(reader* r, header* h) {
	memset(h, 0, sizeof(*h));
	for (;;) {
		uint32_t magic;
		int rc = rd(r, &magic, 4);
		if (rc) return rc;
		if (magic == SHWFS_M_EOD) return 1;
		if ((magic & SHWFS_M_SKIP) == SHWFS_M_SKIP) continue;
		if (magic == SHWFS_M_COMMENT) {
			uint64_t n, n2;
			uint32_t m2;
			if (rd(r, &n, 8)) goto bad;
			if (n > (1u << 30)) goto bad;
			if (n) {
				char* s = (char*)malloc(n);
				if (!s) return err(SHWFS_BIN_ENOMEM, "out of memory", r->path);
				if (rd(r, s, n)) {
					free(s);
					goto bad;
				}
				s[n - 1] = 0;
				if (h->str) {
					char* t = (char*)realloc(h->str, strlen(h->str) + strlen(s) + 1);
					if (!t) {
						free(s);
						return err(SHWFS_BIN_ENOMEM, "out of memory", r->path);
					}
					h->str = t;
					strcat(h->str, s);
					free(s);
				} else {
					h->str = s;
				}
			}
			if (rd(r, &n2, 8) || n2 != n || rd(r, &m2, 4) || m2 != magic) goto bad;
			continue;
		}
		h->id = magic;
		if (rd(r, &h->nx, 8) || rd(r, &h->ny, 8)) goto bad;
		if ((magic & 0x6400u) != 0x6400u) goto bad;
		return 0;
	}
bad:
	free(h->str);
	h->str = NULL;
	return err(SHWFS_BIN_EFORMAT, "bad array header", r->path);
}

static int read_data(reader* r, header* h, shwfs_bin** out);

static int read_cell(reader* r, header* h, shwfs_bin** out) {
	if (h->ny && h->nx > (1ull << 32) / h->ny) {
		free(h->str);
		return err(SHWFS_BIN_EFORMAT, "cell too large", r->path);
	}
	shwfs_bin* c = shwfs_bin_new_cell(h->nx, h->ny, NULL);
	if (!c) return err(SHWFS_BIN_ENOMEM, "out of memory", r->path);
	c->keywords = h->str;
	h->str = NULL;
	for (uint64_t i = 0; i < h->nx * h->ny; i++) {
		header hc;
		int rc = read_header(r, &hc);
		if (rc == 1) break;  // a cell written in part (zfarr) ends early
		if (rc < 0) {
			shwfs_bin_free(c);
			return rc;
		}
		if ((rc = read_data(r, &hc, &c->cells[i]))) {
			shwfs_bin_free(c);
			return rc;
		}
	}
	*out = c;
	return 0;
}

static int read_data(reader* r, header* h, shwfs_bin** out) {
	*out = NULL;
	if (h->id == SHWFS_MCC_ANY) return read_cell(r, h, out);
	const int es = shwfs_bin_elsize(h->id);
	if (!es) {
		free(h->str);
		return err(SHWFS_BIN_EFORMAT, "unsupported array type", r->path);
	}
	if (h->nx == 0 || h->ny == 0) {  // empty member
		free(h->str);
		return 0;
	}
	if (h->nx > (1ull << 40) / h->ny) {
		free(h->str);
		return err(SHWFS_BIN_EFORMAT, "array too large", r->path);
	}
	if (shwfs_bin_is_sparse(h->id)) {
		uint64_t nnz;
		int rc = rd(r, &nnz, 8);
		if (rc || nnz > h->nx * h->ny) {
			free(h->str);
			return rc < 0 ? rc : err(SHWFS_BIN_EFORMAT, "bad sparse matrix", r->path);
		}
		if (nnz == 0) {
			free(h->str);
			return 0;
		}
		shwfs_bin* a = shwfs_bin_new_sparse(h->id, h->nx, h->ny, nnz, NULL, NULL, NULL, NULL);
		if (!a) {
			free(h->str);
			return err(SHWFS_BIN_ENOMEM, "out of memory", r->path);
		}
		a->keywords = h->str;
		h->str = NULL;
		const int iw = sparse_index64(h->id) ? 8 : 4;
		const uint64_t nidx[2] = {h->ny + 1, nnz};
		int64_t* dst[2] = {a->pp, a->pi};
		for (int k = 0; k < 2 && !rc; k++) {
			if (iw == 8) {
				rc = rd(r, dst[k], nidx[k] * 8);
			} else {
				int32_t* t = (int32_t*)malloc(nidx[k] * 4);
				if (!t) rc = err(SHWFS_BIN_ENOMEM, "out of memory", r->path);
				else if (!(rc = rd(r, t, nidx[k] * 4)))
					for (uint64_t i = 0; i < nidx[k]; i++) dst[k][i] = t[i];
				free(t);
			}
		}
		if (!rc) rc = rd(r, a->data, nnz * (uint64_t)es);
		if (!rc && (a->pp[0] != 0 || (uint64_t)a->pp[h->ny] != nnz)) rc = err(SHWFS_BIN_EFORMAT, "bad sparse matrix", r->path);
		if (rc) {
			shwfs_bin_free(a);
			return rc > 0 ? err(SHWFS_BIN_EFORMAT, "truncated file", r->path) : rc;
		}
		*out = a;
		return 0;
	}
	shwfs_bin* a = shwfs_bin_new_dense(h->id, h->nx, h->ny, NULL, NULL);
	if (!a) {
		free(h->str);
		return err(SHWFS_BIN_ENOMEM, "out of memory", r->path);
	}
	a->keywords = h->str;
	h->str = NULL;
	const int rc = rd(r, a->data, h->nx * h->ny * (uint64_t)es);
	if (rc) {
		shwfs_bin_free(a);
		return rc > 0 ? err(SHWFS_BIN_EFORMAT, "truncated file", r->path) : rc;
	}
	*out = a;
	return 0;
}

static int open_reader(reader* r, const char* path) {
	r->path = path;
	r->gz = path ? gzopen(path, "rb") : NULL;
	return r->gz ? 0 : err(SHWFS_BIN_EIO, "cannot open", path);
}

int shwfs_bin_read(const char* path, shwfs_bin** out) {
	if (!out) return err(SHWFS_BIN_EINVAL, "null output", path);
	*out = NULL;
	reader r;
	int rc = open_reader(&r, path);
	if (rc) return rc;
	header h;
	rc = read_header(&r, &h);
	if (rc == 0) rc = read_data(&r, &h, out);
	else if (rc == 1) rc = 0;  // empty file
	gzclose(r.gz);
	return rc;
}

int shwfs_bin_read_all(const char* path, shwfs_bin** out) {
	if (!out) return err(SHWFS_BIN_EINVAL, "null output", path);
	*out = NULL;
	reader r;
	int rc = open_reader(&r, path);
	if (rc) return rc;
	uint64_t n = 0, cap = 8;
	shwfs_bin** v = (shwfs_bin**)calloc(cap, sizeof(shwfs_bin*));
	if (!v) {
		gzclose(r.gz);
		return err(SHWFS_BIN_ENOMEM, "out of memory", path);
	}
	for (;;) {
		header h;
		rc = read_header(&r, &h);
		if (rc) break;
		if (n == cap) {
			shwfs_bin** t = (shwfs_bin**)realloc(v, 2 * cap * sizeof(shwfs_bin*));
			if (!t) {
				rc = err(SHWFS_BIN_ENOMEM, "out of memory", path);
				break;
			}
			v = t;
			cap *= 2;
		}
		if ((rc = read_data(&r, &h, &v[n]))) break;
		n++;
	}
	gzclose(r.gz);
	if (rc < 0) {
		for (uint64_t i = 0; i < n; i++) shwfs_bin_free(v[i]);
		free(v);
		return rc;
	}
	shwfs_bin* c = shwfs_bin_new_cell(n, 1, NULL);
	if (!c) {
		for (uint64_t i = 0; i < n; i++) shwfs_bin_free(v[i]);
		free(v);
		return err(SHWFS_BIN_ENOMEM, "out of memory", path);
	}
	for (uint64_t i = 0; i < n; i++) c->cells[i] = v[i];
	free(v);
	*out = c;
	return 0;
}

/* ---------------------------------------------------------------- writing */
typedef struct {
	FILE* f;
	gzFile gz;
	const char* path;
	int bad;
} writer;

static void wr(writer* w, const void* p, uint64_t n) {
	if (w->bad || !n) return;
	if (w->gz) {
		const char* c = (const char*)p;
		while (n && !w->bad) {
			const unsigned k = n > (1u << 30) ? (1u << 30) : (unsigned)n;
			if (gzwrite(w->gz, c, k) != (int)k) w->bad = 1;
			c += k;
			n -= k;
		}
	} else if (fwrite(p, 1, n, w->f) != n) {
		w->bad = 1;
	}
}

/* write_bin_header (sys/bin.c:762-790) */
static void write_header(writer* w, uint32_t id, uint64_t nx, uint64_t ny, const char* str) {
	if (str) {
		const size_t len = strlen(str);
		const uint64_t n8 = ((len + 8) >> 3) << 3;  // text, NUL and zero padding to 8 bytes
		char* s = (char*)calloc(n8, 1);
		if (!s) {
			w->bad = 1;
			return;
		}
		memcpy(s, str, len);
		const uint32_t mc = SHWFS_M_COMMENT;
		wr(w, &mc, 4);
		wr(w, &n8, 8);
		wr(w, s, n8);
		wr(w, &n8, 8);
		wr(w, &mc, 4);
		free(s);
	}
	const uint32_t ms = SHWFS_M_SKIP;
	wr(w, &ms, 4);
	wr(w, &id, 4);
	wr(w, &nx, 8);
	wr(w, &ny, 8);
}

static void write_data(writer* w, const shwfs_bin* a) {
	if (!a || a->id == SHWFS_MCC_ANY) {  // writedata, math/cell.c:300-328
		const uint64_t n = a ? a->nx * a->ny : 0;
		write_header(w, SHWFS_MCC_ANY, a ? a->nx : 0, a ? a->ny : 0, a ? a->keywords : NULL);
		uint32_t id = 0;
		for (uint64_t i = 0; i < n; i++)
			if (a->cells && a->cells[i]) {
				id = a->cells[i]->id;
				break;
			}
		for (uint64_t i = 0; i < n; i++) {
			if (a->cells && a->cells[i]) write_data(w, a->cells[i]);
			else write_header(w, id, 0, 0, NULL);
		}
		return;
	}
	const int es = shwfs_bin_elsize(a->id);
	if (shwfs_bin_is_sparse(a->id)) {  // spwritedata, math/spbin.c:26-43
		const uint64_t nnz = a->pp ? (uint64_t)a->pp[a->ny] : 0;
		if (!nnz) {
			write_header(w, a->id, 0, 0, NULL);
			return;
		}
		write_header(w, a->id, a->nx, a->ny, a->keywords);
		wr(w, &nnz, 8);
		const uint64_t nidx[2] = {a->ny + 1, nnz};
		const int64_t* src[2] = {a->pp, a->pi};
		for (int k = 0; k < 2; k++) {
			if (sparse_index64(a->id)) {
				wr(w, src[k], nidx[k] * 8);
			} else {
				int32_t* t = (int32_t*)malloc(nidx[k] * 4);
				if (!t) {
					w->bad = 1;
					return;
				}
				for (uint64_t i = 0; i < nidx[k]; i++) t[i] = (int32_t)src[k][i];
				wr(w, t, nidx[k] * 4);
				free(t);
			}
		}
		wr(w, a->data, nnz * (uint64_t)es);
		return;
	}
	write_header(w, a->id, a->nx, a->ny, a->keywords);  // writearr, sys/bin.c:1115-1150
	wr(w, a->data, a->nx * a->ny * (uint64_t)es);
}

static int valid(const shwfs_bin* a) {
	if (!a) return 1;
	if (a->id == SHWFS_MCC_ANY) {
		if (a->nx && a->ny && !a->cells) return 0;
		for (uint64_t i = 0; i < a->nx * a->ny; i++)
			if (!valid(a->cells[i])) return 0;
		return 1;
	}
	if (!shwfs_bin_elsize(a->id)) return 0;
	if (shwfs_bin_is_sparse(a->id)) {
		if (!a->pp) return 1;  // written as an empty matrix
		const uint64_t nnz = (uint64_t)a->pp[a->ny];
		if (a->pp[0] != 0 || (nnz && (!a->pi || !a->data))) return 0;
		for (uint64_t c = 0; c < a->ny; c++)
			if (a->pp[c + 1] < a->pp[c]) return 0;
		for (uint64_t k = 0; k < nnz; k++)
			if (a->pi[k] < 0 || (uint64_t)a->pi[k] >= a->nx) return 0;
		return 1;
	}
	return a->nx * a->ny == 0 || a->data != NULL;
}

int shwfs_bin_write(const char* path, const shwfs_bin* a) {
	if (!path) return err(SHWFS_BIN_EINVAL, "null path", NULL);
	if (!valid(a)) return err(SHWFS_BIN_EINVAL, "inconsistent array", path);
	writer w = {0};
	w.path = path;
	const size_t n = strlen(path);
	if (n > 3 && !strcmp(path + n - 3, ".gz")) w.gz = gzopen(path, "wb");
	else w.f = fopen(path, "wb");
	if (!w.gz && !w.f) return err(SHWFS_BIN_EIO, "cannot open for writing", path);
	write_data(&w, a);
	int bad = w.bad;
	if (w.gz) bad |= gzclose(w.gz) != Z_OK;
	else bad |= fclose(w.f) != 0;
	return bad ? err(SHWFS_BIN_EIO, "write failed", path) : 0;
}
