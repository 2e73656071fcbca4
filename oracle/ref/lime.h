/*
 * lime.h -- a project-written stand-in for the c-lime record library (USQCD
 * c-lime; not part of the reference tree and not installed here), used ONLY to
 * compile the reference's own lib/read_conf_lime.cpp and lib/write_conf_lime.cpp
 * unmodified into the test oracle under oracle/_ref/.  Test infrastructure.
 *
 * It restates the published LIME record format and the c-lime calls those two
 * files make, over the FILE* the caller opened (the reference takes ftell() of
 * that FILE* to find where the binary data starts):
 *   record = 144-byte header, then the data, zero-padded to a multiple of 8;
 *   header = magic 0x456789ab (4 bytes, big-endian), format version 1 (2 bytes),
 *            flags (2 bytes: 0x8000 message begin, 0x4000 message end),
 *            data length (8 bytes, big-endian), record type (128 bytes, NUL-padded).
 * Reader: limeReaderNextRecord moves to the next header (past the current
 * record's padded data) and returns LIME_EOF when none is left;
 * limeReaderReadData reads at most the bytes left in the current record.
 * Writer: limeWriteRecordHeader writes a header; limeWriteRecordData appends
 * data and, when the record's declared length is complete, its zero padding.
 */
#ifndef QKX_REF_LIME_STUB_H
#define QKX_REF_LIME_STUB_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t n_uint64_t; /* as c-lime defines it: unsigned long on LP64 */

#define LIME_SUCCESS 0
#define LIME_EOF 1
#define LIME_ERR_READ (-1)
#define LIME_ERR_WRITE (-2)
#define LIME_ERR_PARAM (-3)

#define QKX_LIME_MAGIC 0x456789abu
#define QKX_LIME_HDR 144

typedef struct {
  FILE* fp;
  long long next;      /* file offset of the next header */
  long long data;      /* file offset of the current record's data */
  n_uint64_t bytes;    /* the current record's data length */
  n_uint64_t done;     /* bytes of it read so far */
  int have;            /* a record is current */
  char type[129];
} LimeReader;

typedef struct {
  int mb, me;
  n_uint64_t bytes;
  char type[129];
} LimeRecordHeader;

typedef struct {
  FILE* fp;
  n_uint64_t bytes;    /* declared length of the record being written */
  n_uint64_t done;     /* data bytes written to it */
} LimeWriter;

static inline n_uint64_t qkx_lime_be(const unsigned char* p, int n) {
  n_uint64_t v = 0;
  for (int i = 0; i < n; i++) v = (v << 8) | p[i];
  return v;
}

static inline void qkx_lime_put(unsigned char* p, n_uint64_t v, int n) {
  for (int i = n - 1; i >= 0; i--) {
    p[i] = (unsigned char)(v & 0xff);
    v >>= 8;
  }
}

static inline n_uint64_t qkx_lime_padded(n_uint64_t n) { return (n + 7) & ~(n_uint64_t)7; }

/* ---------------------------------------------------------------- reader */
static inline LimeReader* limeCreateReader(FILE* fp) {
  if (!fp) return NULL;
  LimeReader* r = (LimeReader*)calloc(1, sizeof(LimeReader));
  if (!r) return NULL;
  r->fp = fp;
  r->next = 0;
  return r;
}

static inline void limeDestroyReader(LimeReader* r) { free(r); }

static inline int limeReaderNextRecord(LimeReader* r) {
  if (!r) return LIME_ERR_PARAM;
  unsigned char h[QKX_LIME_HDR];
  if (fseek(r->fp, (long)r->next, SEEK_SET) != 0) return LIME_EOF;
  const size_t got = fread(h, 1, QKX_LIME_HDR, r->fp);
  if (got == 0) return LIME_EOF;
  if (got != QKX_LIME_HDR) return LIME_ERR_READ;
  if (qkx_lime_be(h, 4) != QKX_LIME_MAGIC) return LIME_ERR_READ;
  r->bytes = qkx_lime_be(h + 8, 8);
  memcpy(r->type, h + 16, 128);
  r->type[128] = 0;
  r->data = r->next + QKX_LIME_HDR;
  r->done = 0;
  r->have = 1;
  r->next = r->data + (long long)qkx_lime_padded(r->bytes);
  return LIME_SUCCESS;
}

static inline char* limeReaderType(LimeReader* r) { return r && r->have ? r->type : NULL; }

static inline n_uint64_t limeReaderBytes(LimeReader* r) { return r && r->have ? r->bytes : 0; }

static inline int limeReaderReadData(void* dest, n_uint64_t* nbytes, LimeReader* r) {
  if (!r || !r->have || !nbytes) return LIME_ERR_PARAM;
  n_uint64_t want = *nbytes, left = r->bytes - r->done;
  if (want > left) want = left;
  if (fseek(r->fp, (long)(r->data + (long long)r->done), SEEK_SET) != 0) return LIME_ERR_READ;
  const size_t got = fread(dest, 1, (size_t)want, r->fp);
  r->done += got;
  *nbytes = got;
  return got == want ? LIME_SUCCESS : LIME_ERR_READ;
}

/* ---------------------------------------------------------------- writer */
static inline LimeWriter* limeCreateWriter(FILE* fp) {
  if (!fp) return NULL;
  LimeWriter* w = (LimeWriter*)calloc(1, sizeof(LimeWriter));
  if (w) w->fp = fp;
  return w;
}

static inline void limeDestroyWriter(LimeWriter* w) { free(w); }

static inline LimeRecordHeader* limeCreateHeader(int MB_flag, int ME_flag, char* type, n_uint64_t reclen) {
  LimeRecordHeader* h = (LimeRecordHeader*)calloc(1, sizeof(LimeRecordHeader));
  if (!h) return NULL;
  h->mb = MB_flag;
  h->me = ME_flag;
  h->bytes = reclen;
  strncpy(h->type, type, 128);
  return h;
}

static inline void limeDestroyHeader(LimeRecordHeader* h) { free(h); }

static inline int limeWriteRecordHeader(LimeRecordHeader* h, LimeWriter* w) {
  if (!h || !w) return LIME_ERR_PARAM;
  unsigned char b[QKX_LIME_HDR];
  memset(b, 0, sizeof b);
  qkx_lime_put(b, QKX_LIME_MAGIC, 4);
  qkx_lime_put(b + 4, 1, 2);
  qkx_lime_put(b + 6, (h->mb ? 0x8000u : 0u) | (h->me ? 0x4000u : 0u), 2);
  qkx_lime_put(b + 8, h->bytes, 8);
  memcpy(b + 16, h->type, strlen(h->type) < 128 ? strlen(h->type) : 128);
  if (fwrite(b, 1, QKX_LIME_HDR, w->fp) != QKX_LIME_HDR) return LIME_ERR_WRITE;
  w->bytes = h->bytes;
  w->done = 0;
  return LIME_SUCCESS;
}

static inline int limeWriteRecordData(void* src, n_uint64_t* nbytes, LimeWriter* w) {
  if (!w || !nbytes) return LIME_ERR_PARAM;
  n_uint64_t n = *nbytes, left = w->bytes - w->done;
  if (n > left) n = left;
  if (n && fwrite(src, 1, (size_t)n, w->fp) != n) return LIME_ERR_WRITE;
  w->done += n;
  *nbytes = n;
  if (w->done == w->bytes) {
    static const unsigned char zeros[8] = {0};
    const size_t pad = (size_t)(qkx_lime_padded(w->bytes) - w->bytes);
    if (pad && fwrite(zeros, 1, pad, w->fp) != pad) return LIME_ERR_WRITE;
  }
  return LIME_SUCCESS;
}

#endif
