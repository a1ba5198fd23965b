/*
 * Checkpoint files in the reference's HDF5 layout, without an HDF5 library.
 *
 * io_hdf5_out (src/IO/io_hdf5.c:15-159) creates a file with default property
 * lists and writes three datasets of H5T_NATIVE_DOUBLE into its root group:
 * "T" [1], "GravMass" [2][4] and "Data" [Ncells_global][NUM_Q+3], the last
 * with contiguous storage (its H5Pset_chunk is commented out, :121).
 * io_hdf5_in (:161-266) opens input.h5 and reads the three back, "Data" as the
 * hyperslab of rows [sim_offset, sim_offset + Ncells).
 *
 * This file writes and reads such files by the HDF5 file format
 * specification, with the structures the library writes by default under its
 * earliest format bounds:
 *   - superblock version 0 at address 0, 8-byte offsets and lengths, group
 *     leaf-node K 4, group internal-node K 16;
 *   - the root group as a symbol table: a version-1 object header holding a
 *     symbol-table message, a local heap of link names, a version-1 B-tree of
 *     type 0 with one leaf, and one symbol-table node (SNOD) whose entries are
 *     sorted by name;
 *   - per dataset a version-1 object header with a dataspace message
 *     (version 1), a datatype message (version 1: IEEE 754 binary64, little
 *     endian), a fill-value message (version 2: late allocation, written if
 *     set, default value) and a layout message (version 3, contiguous), and
 *     the raw values after the headers.
 *
 * The reader accepts what the library may have written in those formats: a
 * user block before the superblock (the signature is searched at 0 and at
 * 512, 1024, 2048, ...), superblock version 1, B-tree internal nodes and
 * several symbol-table nodes, object-header continuation blocks, messages it
 * does not need, dataspace version 2, and layout versions 1-3 (contiguous;
 * compact in version 3).  Datasets must hold 64-bit little-endian IEEE
 * floats.  Version-2 object headers and superblock versions 2-3 (the
 * library's "latest" format) are refused with an error.
 */
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dgpu_h5.h"

#define H5_UNDEF UINT64_MAX
static const unsigned char h5_sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

enum {
  H5M_NIL = 0x0000,
  H5M_DATASPACE = 0x0001,
  H5M_DATATYPE = 0x0003,
  H5M_FILL = 0x0005,
  H5M_LAYOUT = 0x0008,
  H5M_CONT = 0x0010,
  H5M_STAB = 0x0011,
};

enum { LEAF_K = 4, INTERNAL_K = 16 };
#define SB_SIZE 96u                                  /* superblock version 0 */
#define OH_PREFIX 16u                                /* version-1 object header prefix, aligned */
#define HEAP_HDR 32u                                 /* "HEAP" header */
#define BTREE_SIZE (24u + 2u * INTERNAL_K * 8u + (2u * INTERNAL_K + 1u) * 8u)
#define SNOD_SIZE (8u + 2u * LEAF_K * 40u)

/* ------------------------------------------------------------------ writer */

typedef struct {
  unsigned char *p;
  size_t n, cap;
  int oom;
} wbuf;

static void w_reserve(wbuf *b, size_t n) {
  if (b->oom || n <= b->cap) return;
  size_t c = b->cap ? b->cap : 4096;
  while (c < n) c *= 2;
  unsigned char *q = (unsigned char *)realloc(b->p, c);
  if (!q) {
    b->oom = 1;
    return;
  }
  memset(q + b->cap, 0, c - b->cap);
  b->p = q;
  b->cap = c;
}

/* little-endian store of the low `len` bytes of v at absolute offset `at` */
static void w_at(wbuf *b, size_t at, uint64_t v, int len) {
  int k;
  w_reserve(b, at + (size_t)len);
  if (b->oom) return;
  for (k = 0; k < len; ++k) b->p[at + (size_t)k] = (unsigned char)(v >> (8 * k));
  if (at + (size_t)len > b->n) b->n = at + (size_t)len;
}

static void w_bytes(wbuf *b, size_t at, const void *src, size_t len) {
  w_reserve(b, at + len);
  if (b->oom) return;
  memcpy(b->p + at, src, len);
  if (at + len > b->n) b->n = at + len;
}

/* one message of a version-1 object header: 8-byte header, body padded to 8 */
static size_t w_msg(wbuf *b, size_t at, int type, int flags, size_t body) {
  w_at(b, at, (uint64_t)type, 2);
  w_at(b, at + 2, (uint64_t)body, 2);
  w_at(b, at + 4, (uint64_t)flags, 1);
  return at + 8;
}

static size_t pad8(size_t n) { return (n + 7u) & ~(size_t)7u; }

/* size of a dataset's object header (prefix + four messages) */
static size_t oh_dset_size(int rank) {
  return OH_PREFIX + (8 + pad8(8 + 8 * (size_t)rank)) + (8 + 24) + (8 + 8) + (8 + 24);
}

static void w_dset_header(wbuf *b, size_t at, int rank, const uint64_t *dims, uint64_t data_addr) {
  const size_t total = oh_dset_size(rank);
  size_t m = at + OH_PREFIX, q;
  int r;
  uint64_t nbytes = 8;
  for (r = 0; r < rank; ++r) nbytes *= dims[r];
  /* prefix: version 1, 4 messages, reference count 1, chunk size */
  w_at(b, at, 1, 1);
  w_at(b, at + 2, 4, 2);
  w_at(b, at + 4, 1, 4);
  w_at(b, at + 8, (uint64_t)(total - OH_PREFIX), 4);
  /* dataspace, version 1: rank, no maximum dimensions */
  q = w_msg(b, m, H5M_DATASPACE, 0, pad8(8 + 8 * (size_t)rank));
  w_at(b, q, 1, 1);
  w_at(b, q + 1, (uint64_t)rank, 1);
  for (r = 0; r < rank; ++r) w_at(b, q + 8 + 8 * (size_t)r, dims[r], 8);
  m = q + pad8(8 + 8 * (size_t)rank);
  /* datatype, version 1, class 1 (floating point): little endian, mantissa
   * normalisation "implied", sign bit 63; size 8; offset 0, precision 64,
   * exponent at 52 of 11 bits, mantissa at 0 of 52 bits, bias 1023 */
  q = w_msg(b, m, H5M_DATATYPE, 1, 24);
  w_at(b, q, 0x11, 1);
  w_at(b, q + 1, 0x20, 1);
  w_at(b, q + 2, 63, 1);
  w_at(b, q + 3, 0, 1);
  w_at(b, q + 4, 8, 4);
  w_at(b, q + 8, 0, 2);
  w_at(b, q + 10, 64, 2);
  w_at(b, q + 12, 52, 1);
  w_at(b, q + 13, 11, 1);
  w_at(b, q + 14, 0, 1);
  w_at(b, q + 15, 52, 1);
  w_at(b, q + 16, 1023, 4);
  m = q + 24;
  /* fill value, version 2: allocation late (2), fill written if set (2),
   * defined (1) with size 0: the library's default value */
  q = w_msg(b, m, H5M_FILL, 1, 8);
  w_at(b, q, 2, 1);
  w_at(b, q + 1, 2, 1);
  w_at(b, q + 2, 2, 1);
  w_at(b, q + 3, 1, 1);
  w_at(b, q + 4, 0, 4);
  m = q + 8;
  /* layout, version 3, class 1 (contiguous): address and size */
  q = w_msg(b, m, H5M_LAYOUT, 0, 24);
  w_at(b, q, 3, 1);
  w_at(b, q + 1, 1, 1);
  w_at(b, q + 2, data_addr, 8);
  w_at(b, q + 10, nbytes, 8);
  m = q + 24;
  (void)m;
}

int h5_write(const char *path, const h5_dataset *ds, int n, char *err, int errlen) {
  /* names sorted by strcmp, as a symbol-table node keeps them */
  int order[2 * LEAF_K], i, j;
  size_t heap_off[2 * LEAF_K], heap_size = 8, oh_addr[2 * LEAF_K];
  uint64_t data_addr[2 * LEAF_K];
  wbuf b = {0};
  FILE *f;
  if (n < 1 || n > 2 * LEAF_K) return snprintf(err, (size_t)errlen, "between 1 and %d datasets", 2 * LEAF_K), -1;
  for (i = 0; i < n; ++i) {
    if (ds[i].rank < 1 || ds[i].rank > 2 || !ds[i].name || !ds[i].name[0])
      return snprintf(err, (size_t)errlen, "dataset %d: rank 1 or 2 and a name", i), -1;
    order[i] = i;
  }
  for (i = 1; i < n; ++i)
    for (j = i; j > 0 && strcmp(ds[order[j - 1]].name, ds[order[j]].name) > 0; --j) {
      int t = order[j];
      order[j] = order[j - 1];
      order[j - 1] = t;
    }
  for (i = 1; i < n; ++i)
    if (!strcmp(ds[order[i - 1]].name, ds[order[i]].name))
      return snprintf(err, (size_t)errlen, "duplicate dataset name %s", ds[order[i]].name), -1;
  /* local heap: "" at 0 (the root's own link name), then each name */
  for (i = 0; i < n; ++i) {
    heap_off[order[i]] = heap_size;
    heap_size += pad8(strlen(ds[order[i]].name) + 1);
  }
  const size_t a_root = SB_SIZE, root_size = OH_PREFIX + 8 + 16;
  const size_t a_heap = a_root + root_size, a_heapdata = a_heap + HEAP_HDR;
  const size_t a_btree = a_heapdata + heap_size, a_snod = a_btree + BTREE_SIZE;
  size_t a = a_snod + SNOD_SIZE;
  for (i = 0; i < n; ++i) {
    oh_addr[i] = a;
    a += oh_dset_size(ds[i].rank);
  }
  for (i = 0; i < n; ++i) {
    uint64_t cnt = 1;
    int r;
    for (r = 0; r < ds[i].rank; ++r) cnt *= ds[i].dims[r];
    data_addr[i] = a;
    a += (size_t)(8 * cnt);
  }
  const uint64_t eof = a;

  /* superblock version 0 */
  w_bytes(&b, 0, h5_sig, 8);
  w_at(&b, 13, 8, 1);  /* size of offsets */
  w_at(&b, 14, 8, 1);  /* size of lengths */
  w_at(&b, 16, LEAF_K, 2);
  w_at(&b, 18, INTERNAL_K, 2);
  w_at(&b, 24, 0, 8);          /* base address */
  w_at(&b, 32, H5_UNDEF, 8);   /* free-space info */
  w_at(&b, 40, eof, 8);        /* end of file */
  w_at(&b, 48, H5_UNDEF, 8);   /* driver information */
  /* root symbol-table entry: name offset 0, header, cache type 1 with the
   * B-tree and heap addresses in the scratch pad */
  w_at(&b, 56, 0, 8);
  w_at(&b, 64, a_root, 8);
  w_at(&b, 72, 1, 4);
  w_at(&b, 80, a_btree, 8);
  w_at(&b, 88, a_heap, 8);

  /* root object header: one symbol-table message */
  w_at(&b, a_root, 1, 1);
  w_at(&b, a_root + 2, 1, 2);
  w_at(&b, a_root + 4, 1, 4);
  w_at(&b, a_root + 8, root_size - OH_PREFIX, 4);
  {
    size_t q = w_msg(&b, a_root + OH_PREFIX, H5M_STAB, 0, 16);
    w_at(&b, q, a_btree, 8);
    w_at(&b, q + 8, a_heap, 8);
  }

  /* local heap: no free block (head of the free list: 1, "none") */
  w_bytes(&b, a_heap, "HEAP", 4);
  w_at(&b, a_heap + 8, heap_size, 8);
  w_at(&b, a_heap + 16, 1, 8);
  w_at(&b, a_heap + 24, a_heapdata, 8);
  w_at(&b, a_heapdata + heap_size - 1, 0, 1);
  for (i = 0; i < n; ++i) w_bytes(&b, a_heapdata + heap_off[i], ds[i].name, strlen(ds[i].name));

  /* B-tree leaf (type 0, level 0, one child): keys are heap offsets, the
   * right key that of the last name of the node */
  w_bytes(&b, a_btree, "TREE", 4);
  w_at(&b, a_btree + 6, 1, 2);
  w_at(&b, a_btree + 8, H5_UNDEF, 8);
  w_at(&b, a_btree + 16, H5_UNDEF, 8);
  w_at(&b, a_btree + 24, 0, 8);
  w_at(&b, a_btree + 32, a_snod, 8);
  w_at(&b, a_btree + 40, heap_off[order[n - 1]], 8);
  w_at(&b, a_btree + BTREE_SIZE - 1, 0, 1);

  /* symbol-table node */
  w_bytes(&b, a_snod, "SNOD", 4);
  w_at(&b, a_snod + 4, 1, 1);
  w_at(&b, a_snod + 6, (uint64_t)n, 2);
  for (i = 0; i < n; ++i) {
    const size_t e = a_snod + 8 + 40 * (size_t)i;
    w_at(&b, e, heap_off[order[i]], 8);
    w_at(&b, e + 8, oh_addr[order[i]], 8);
  }
  w_at(&b, a_snod + SNOD_SIZE - 1, 0, 1);

  for (i = 0; i < n; ++i) {
    uint64_t cnt = 1;
    int r;
    w_dset_header(&b, oh_addr[i], ds[i].rank, ds[i].dims, data_addr[i]);
    for (r = 0; r < ds[i].rank; ++r) cnt *= ds[i].dims[r];
    if (cnt) w_bytes(&b, (size_t)data_addr[i], ds[i].data, (size_t)(8 * cnt));
  }
  if (b.oom || b.n != (size_t)eof) {
    free(b.p);
    return snprintf(err, (size_t)errlen, "%s", b.oom ? "out of host memory" : "internal size mismatch"), -2;
  }
  f = fopen(path, "wb");
  if (!f) {
    free(b.p);
    return snprintf(err, (size_t)errlen, "cannot create %s: %s", path, strerror(errno)), -1;
  }
  if (fwrite(b.p, 1, b.n, f) != b.n || fclose(f) != 0) {
    free(b.p);
    return snprintf(err, (size_t)errlen, "cannot write %s", path), -1;
  }
  free(b.p);
  return 0;
}

/* ------------------------------------------------------------------ reader */

typedef struct {
  const unsigned char *p;
  uint64_t n;    /* file size */
  uint64_t base; /* absolute address of the superblock's base */
  char *err;
  int errlen;
} rfile;

static int r_fail(rfile *f, const char *msg, uint64_t at) {
  snprintf(f->err, (size_t)f->errlen, "%s (at byte %llu)", msg, (unsigned long long)at);
  return -1;
}

/* bytes [a, a+len) of the file, addresses relative to the base; NULL if out */
static const unsigned char *r_ptr(rfile *f, uint64_t a, uint64_t len) {
  if (a == H5_UNDEF || a > UINT64_MAX - f->base) return NULL;
  a += f->base;
  if (a > f->n || len > f->n - a) return NULL;
  return f->p + a;
}

static uint64_t le(const unsigned char *q, int len) {
  uint64_t v = 0;
  int k;
  for (k = len - 1; k >= 0; --k) v = (v << 8) | q[k];
  return v;
}

typedef struct {
  int rank;
  uint64_t dims[H5_MAX_RANK];
  int have_space, have_type, have_layout;
  int compact;
  uint64_t addr, size;          /* contiguous storage */
  const unsigned char *inline_; /* compact storage */
  uint64_t btree, heap;         /* symbol-table message */
  int have_stab;
} ohinfo;

static int r_message(rfile *f, int type, const unsigned char *q, uint64_t len, uint64_t at, ohinfo *o) {
  if (type == H5M_DATASPACE) {
    int ver, rank, r;
    size_t off;
    if (len < 8) return r_fail(f, "short dataspace message", at);
    ver = q[0];
    rank = q[1];
    if (ver == 1) off = 8;
    else if (ver == 2) off = 4;
    else return r_fail(f, "unsupported dataspace message version", at);
    if (rank > H5_MAX_RANK) return r_fail(f, "dataspace rank above 2", at);
    if (off + 8u * (uint64_t)rank > len) return r_fail(f, "short dataspace message", at);
    if (ver == 2 && q[3] == 2) return r_fail(f, "null dataspace", at);
    o->rank = rank;
    for (r = 0; r < rank; ++r) o->dims[r] = le(q + off + 8 * (size_t)r, 8);
    o->have_space = 1;
  } else if (type == H5M_DATATYPE) {
    if (len < 20) return r_fail(f, "short datatype message", at);
    if ((q[0] & 0x0f) != 1 || le(q + 4, 4) != 8 || (q[1] & 0x01) || le(q + 8, 2) != 0 ||
        le(q + 10, 2) != 64 || q[12] != 52 || q[13] != 11 || q[14] != 0 || q[15] != 52 ||
        le(q + 16, 4) != 1023 || q[2] != 63)
      return r_fail(f, "dataset is not 64-bit little-endian IEEE floating point", at);
    o->have_type = 1;
  } else if (type == H5M_LAYOUT) {
    int ver = len ? q[0] : 0;
    if (ver == 1 || ver == 2) {
      int nd, cls, d;
      uint64_t sz = 1;
      if (len < 8) return r_fail(f, "short layout message", at);
      nd = q[1];
      cls = q[2];
      if (cls != 1) return r_fail(f, "only contiguous storage is read from layout versions 1-2", at);
      if (len < 16 + 4u * (uint64_t)nd) return r_fail(f, "short layout message", at);
      o->addr = le(q + 8, 8);
      for (d = 0; d < nd; ++d) sz *= le(q + 16 + 4 * (size_t)d, 4);
      o->size = sz;
    } else if (ver == 3) {
      if (len < 2) return r_fail(f, "short layout message", at);
      if (q[1] == 1) {
        if (len < 18) return r_fail(f, "short layout message", at);
        o->addr = le(q + 2, 8);
        o->size = le(q + 10, 8);
      } else if (q[1] == 0) {
        if (len < 4) return r_fail(f, "short layout message", at);
        o->size = le(q + 2, 2);
        if (4 + o->size > len) return r_fail(f, "short compact layout message", at);
        o->inline_ = q + 4;
        o->compact = 1;
      } else {
        return r_fail(f, "chunked storage is not read here", at);
      }
    } else {
      return r_fail(f, "unsupported layout message version", at);
    }
    o->have_layout = 1;
  } else if (type == H5M_STAB) {
    if (len < 16) return r_fail(f, "short symbol-table message", at);
    o->btree = le(q, 8);
    o->heap = le(q + 8, 8);
    o->have_stab = 1;
  }
  return 0;
}

/* version-1 object header at address a, continuation blocks included */
static int r_header(rfile *f, uint64_t a, ohinfo *o) {
  const unsigned char *h = r_ptr(f, a, OH_PREFIX);
  uint64_t chunk, clen;
  unsigned nmsg, seen = 0;
  int nchunks = 0;
  uint64_t conts[64][2];
  int ncont = 0;
  memset(o, 0, sizeof(*o));
  if (!h) return r_fail(f, "object header outside the file", a);
  if (h[0] != 1) return r_fail(f, "only version-1 object headers are read here", a);
  nmsg = (unsigned)le(h + 2, 2);
  chunk = a + OH_PREFIX;
  clen = le(h + 8, 4);
  for (;;) {
    uint64_t pos = 0;
    if (++nchunks > 64) return r_fail(f, "too many object header continuation blocks", a);
    while (pos + 8 <= clen && seen < nmsg) {
      const unsigned char *m = r_ptr(f, chunk + pos, 8);
      const unsigned char *body;
      int type;
      uint64_t len;
      if (!m) return r_fail(f, "object header message outside the file", chunk + pos);
      type = (int)le(m, 2);
      len = le(m + 2, 2);
      body = r_ptr(f, chunk + pos + 8, len);
      if (!body || pos + 8 + len > clen) return r_fail(f, "object header message overruns its block", chunk + pos);
      if (m[4] & 0x02) return r_fail(f, "shared object header messages are not read here", chunk + pos);
      if (type == H5M_CONT) {
        if (len < 16 || ncont == 64) return r_fail(f, "bad continuation message", chunk + pos);
        conts[ncont][0] = le(body, 8);
        conts[ncont][1] = le(body + 8, 8);
        ++ncont;
      } else if (r_message(f, type, body, len, chunk + pos, o)) {
        return -1;
      }
      ++seen;
      pos += 8 + len;
    }
    if (seen >= nmsg || ncont == 0) break;
    chunk = conts[0][0];
    clen = conts[0][1];
    memmove(conts[0], conts[1], sizeof(conts[0]) * (size_t)(ncont - 1));
    --ncont;
  }
  return 0;
}

typedef struct {
  const char *name;
  uint64_t found;
} lookup;

/* walks a group B-tree (type 0) down to its symbol-table nodes */
static int r_btree(rfile *f, uint64_t a, const unsigned char *heap, uint64_t heapsize, lookup *lk, int depth) {
  const unsigned char *t = r_ptr(f, a, 24);
  unsigned used, c;
  int level;
  if (depth > 32) return r_fail(f, "B-tree too deep", a);
  if (!t || memcmp(t, "TREE", 4)) return r_fail(f, "missing B-tree node", a);
  if (t[4] != 0) return r_fail(f, "B-tree is not a group B-tree", a);
  level = t[5];
  used = (unsigned)le(t + 6, 2);
  if (!r_ptr(f, a + 24, 16u * (uint64_t)used + 8)) return r_fail(f, "B-tree node outside the file", a);
  for (c = 0; c < used && lk->found == H5_UNDEF; ++c) {
    const uint64_t child = le(r_ptr(f, a + 24 + 16u * c + 8, 8), 8);
    if (level > 0) {
      if (r_btree(f, child, heap, heapsize, lk, depth + 1)) return -1;
    } else {
      const unsigned char *s = r_ptr(f, child, 8);
      unsigned ns, e;
      if (!s || memcmp(s, "SNOD", 4)) return r_fail(f, "missing symbol-table node", child);
      ns = (unsigned)le(s + 6, 2);
      if (!r_ptr(f, child + 8, 40u * (uint64_t)ns)) return r_fail(f, "symbol-table node outside the file", child);
      for (e = 0; e < ns; ++e) {
        const unsigned char *en = r_ptr(f, child + 8 + 40u * e, 40);
        const uint64_t off = le(en, 8);
        if (off >= heapsize) return r_fail(f, "link name outside the local heap", child);
        if (strnlen((const char *)heap + off, (size_t)(heapsize - off)) < heapsize - off &&
            !strcmp((const char *)heap + off, lk->name)) {
          lk->found = le(en + 8, 8);
          break;
        }
      }
    }
  }
  return 0;
}

static int r_open(rfile *f, const unsigned char *p, uint64_t n, uint64_t *root) {
  uint64_t off;
  const unsigned char *sb = NULL;
  size_t entry;
  f->p = p;
  f->n = n;
  f->base = 0;
  for (off = 0; off + 8 <= n; off = off ? 2 * off : 512)
    if (!memcmp(p + off, h5_sig, 8)) {
      sb = p + off;
      break;
    }
  if (!sb) return r_fail(f, "not an HDF5 file (no superblock signature)", 0);
  if (n - off < 100) return r_fail(f, "truncated superblock", off);
  if (sb[8] > 1) return r_fail(f, "superblock versions 2-3 are not read here", off);
  if (sb[13] != 8 || sb[14] != 8) return r_fail(f, "only 8-byte offsets and lengths are read here", off);
  entry = sb[8] == 0 ? 56 : 60;
  f->base = le(sb + entry - 32, 8);
  if (f->base > n) return r_fail(f, "base address outside the file", off);
  *root = le(sb + entry + 8, 8);
  return 0;
}

int h5_read(const char *path, const char *name, int *rank, uint64_t *dims, double *data,
            uint64_t row0, uint64_t nrows, char *err, int errlen) {
  FILE *fp = fopen(path, "rb");
  unsigned char *buf = NULL;
  long sz;
  uint64_t root;
  rfile f;
  ohinfo o;
  int rc = -1;
  f.err = err;
  f.errlen = errlen;
  if (!fp) return snprintf(err, (size_t)errlen, "cannot open %s: %s", path, strerror(errno)), -1;
  if (fseek(fp, 0, SEEK_END) || (sz = ftell(fp)) < 0 || fseek(fp, 0, SEEK_SET)) {
    fclose(fp);
    return snprintf(err, (size_t)errlen, "cannot size %s", path), -1;
  }
  buf = (unsigned char *)malloc((size_t)sz + 1);
  if (!buf || fread(buf, 1, (size_t)sz, fp) != (size_t)sz) {
    fclose(fp);
    free(buf);
    return snprintf(err, (size_t)errlen, "cannot read %s", path), -1;
  }
  fclose(fp);
  if (r_open(&f, buf, (uint64_t)sz, &root)) goto out;
  if (r_header(&f, root, &o)) goto out;
  if (!o.have_stab) {
    r_fail(&f, "root group has no symbol table (a newer-format group)", root);
    goto out;
  }
  {
    const unsigned char *hh = r_ptr(&f, o.heap, 32);
    const unsigned char *heap;
    uint64_t hsize;
    lookup lk = {name, H5_UNDEF};
    if (!hh || memcmp(hh, "HEAP", 4)) {
      r_fail(&f, "missing local heap", o.heap);
      goto out;
    }
    hsize = le(hh + 8, 8);
    heap = r_ptr(&f, le(hh + 24, 8), hsize);
    if (!heap) {
      r_fail(&f, "local heap data outside the file", o.heap);
      goto out;
    }
    if (r_btree(&f, o.btree, heap, hsize, &lk, 0)) goto out;
    if (lk.found == H5_UNDEF) {
      snprintf(err, (size_t)errlen, "no dataset %s in %s", name, path);
      goto out;
    }
    if (r_header(&f, lk.found, &o)) goto out;
  }
  if (!o.have_space || !o.have_type || !o.have_layout) {
    r_fail(&f, "dataset header lacks a dataspace, datatype or layout message", 0);
    goto out;
  }
  {
    uint64_t cnt = 1, rowlen = 1;
    int r;
    for (r = 0; r < o.rank; ++r) cnt *= o.dims[r];
    for (r = 1; r < o.rank; ++r) rowlen *= o.dims[r];
    if (o.size != 8 * cnt) {
      r_fail(&f, "stored size differs from the dataspace", 0);
      goto out;
    }
    *rank = o.rank;
    for (r = 0; r < o.rank; ++r) dims[r] = o.dims[r];
    if (data) {
      const unsigned char *src;
      const uint64_t rows = o.rank ? o.dims[0] : 1;
      if (row0 > rows || nrows > rows - row0) {
        snprintf(err, (size_t)errlen, "%s: rows [%llu, %llu) outside its %llu rows", name,
                 (unsigned long long)row0, (unsigned long long)(row0 + nrows), (unsigned long long)rows);
        goto out;
      }
      if (o.compact) src = o.inline_;
      else if (!(src = r_ptr(&f, o.addr, o.size))) {
        r_fail(&f, "dataset values outside the file", o.addr);
        goto out;
      }
      memcpy(data, src + 8 * row0 * rowlen, (size_t)(8 * nrows * rowlen));
    }
  }
  rc = 0;
out:
  free(buf);
  return rc;
}
