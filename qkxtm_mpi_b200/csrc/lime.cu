// lime.cu -- ILDG gauge configurations in LIME files: the reader of
// lib/read_conf_lime.cpp (qkxTM_MPI_getGaugeLime) and the writer of
// lib/write_conf_lime.cpp (qkxTM_writeGaugeLime), without c-lime.
//
// LIME record (the published c-lime format): a 144-byte big-endian header
//   [0,4)   magic number 0x456789ab
//   [4,6)   version (1)
//   [6,8)   flags: bit 15 message begin (MB), bit 14 message end (ME)
//   [8,16)  data length in bytes
//   [16,144) record type, NUL-padded ASCII
// then the data, padded with zeros to a multiple of 8 bytes.
//
// The host parses the headers and streams the binary record through two
// page-locked buffers (disk reads overlap the copies to the device); the GPU
// swaps the bytes and lays the links out for the operator.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "layout.cuh"
#include "qkx_ctx.cuh"

using namespace qkx;

namespace qkx {
namespace {

constexpr uint32_t LIME_MAGIC = 0x456789abu;
constexpr size_t LIME_HDR = 144;
constexpr size_t LIME_CHUNK = (size_t)64 << 20;  // bytes per streamed chunk

int bad(const char* fmt, const char* arg = "") {
  set_error(fmt, arg);
  return QKX_ERR_INVALID;
}

uint64_t be64(const unsigned char* p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; i++) v = (v << 8) | p[i];
  return v;
}
uint32_t be32(const unsigned char* p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }
void put_be64(unsigned char* p, uint64_t v) {
  for (int i = 7; i >= 0; i--) {
    p[i] = (unsigned char)(v & 0xff);
    v >>= 8;
  }
}

struct LimeRecord {
  uint64_t offset;  // of the data
  uint64_t bytes;
  std::string type;
};

// scan every record header of the file
int lime_scan(FILE* f, std::vector<LimeRecord>& recs) {
  if (fseeko(f, 0, SEEK_END) != 0) return bad("cannot seek in the LIME file%s");
  const uint64_t size = (uint64_t)ftello(f);
  uint64_t pos = 0;
  while (pos + LIME_HDR <= size) {
    unsigned char h[LIME_HDR];
    if (fseeko(f, (off_t)pos, SEEK_SET) != 0 || fread(h, 1, LIME_HDR, f) != LIME_HDR)
      return bad("short read of a LIME header%s");
    if (be32(h) != LIME_MAGIC) return bad("not a LIME record (bad magic number)%s");
    LimeRecord r;
    r.offset = pos + LIME_HDR;
    r.bytes = be64(h + 8);
    char t[129];
    memcpy(t, h + 16, 128);
    t[128] = 0;
    r.type = t;
    // r.offset <= size here, so size - r.offset cannot wrap; once r.bytes fits,
    // its 8-byte padded length cannot overflow either
    if (r.bytes > size - r.offset) return bad("LIME record '%s' runs past the end of the file", r.type.c_str());
    recs.push_back(r);
    pos = r.offset + ((r.bytes + 7) & ~(uint64_t)7);
  }
  if (pos != size && pos + LIME_HDR > size && pos < size) return bad("trailing bytes after the last LIME record%s");
  return QKX_OK;
}

// integer after <tag> in an XML text (spaces allowed), or -1
long xml_int(const std::string& xml, const char* tag) {
  const size_t i = xml.find(tag);
  if (i == std::string::npos) return -1;
  long v = -1;
  if (sscanf(xml.c_str() + i + strlen(tag), " %ld", &v) != 1) return -1;
  return v;
}

// big-endian 8-byte words -> native doubles (n words)
__global__ void k_bswap64(const unsigned long long* __restrict__ in, double* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = __longlong_as_double((long long)__byte_perm((unsigned)(in[i] >> 32), 0, 0x0123) |
                                  ((long long)__byte_perm((unsigned)in[i], 0, 0x0123) << 32));
}

// big-endian 4-byte words -> native floats, widened to double
__global__ void k_bswap32(const unsigned* __restrict__ in, double* __restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)__uint_as_float(__byte_perm(in[i], 0, 0x0123));
}

int swap_grid(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace
}  // namespace qkx

extern "C" {

int qkx_read_gauge_lime(qkx_ctx* c, const char* path, int bc_mode, double* U_host, qkx_lime_info* info) {
  if (!c || !path) return bad("invalid argument: NULL argument%s");
  if (bc_mode != QKX_LINKS_AS_GIVEN && bc_mode != QKX_LINKS_APPLY_BC) return bad("invalid argument: bc_mode%s");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_links(c));
  FILE* f = fopen(path, "rb");
  if (!f) return bad("cannot open '%s' for reading", path);
  std::vector<LimeRecord> recs;
  int rc = lime_scan(f, recs);
  int precision = 64, L[4] = {0, 0, 0, 0};
  const LimeRecord* bin = nullptr;
  for (const LimeRecord& r : recs) {
    if (rc != QKX_OK) break;
    if (r.type == "ildg-format" && r.bytes < (1u << 20)) {
      std::string xml(r.bytes, '\0');
      if (fseeko(f, (off_t)r.offset, SEEK_SET) != 0 || fread(&xml[0], 1, r.bytes, f) != r.bytes) {
        rc = bad("short read of the ildg-format record%s");
        break;
      }
      precision = (int)xml_int(xml, "<precision>");
      const char* tags[4] = {"<lx>", "<ly>", "<lz>", "<lt>"};
      for (int i = 0; i < 4; i++) L[i] = (int)std::max<long>(0, xml_int(xml, tags[i]));
    }
    if (r.type == "ildg-binary-data") {
      bin = &r;
      break;  // as the reference: the first binary record is the configuration
    }
  }
  if (rc == QKX_OK && !bin) rc = bad("no ildg-binary-data record in '%s'", path);
  if (rc == QKX_OK && precision != 64 && precision != 32) rc = bad("unknown precision in the ildg-format record%s");
  for (int i = 0; i < 4 && rc == QKX_OK; i++)
    if (L[i] != 0 && L[i] != c->p.L[i]) rc = bad("the file's lattice extents differ from the context's%s");
  const size_t nwords = (size_t)72 * c->V;  // reals
  const size_t wsize = precision == 64 ? 8 : 4;
  if (rc == QKX_OK && bin->bytes != nwords * wsize) rc = bad("the binary record has the wrong size for this lattice%s");
  if (info) {
    info->precision = precision;
    for (int i = 0; i < 4; i++) info->L[i] = L[i];
    info->data_offset = bin ? (long long)bin->offset : -1;
    info->data_bytes = bin ? (long long)bin->bytes : 0;
    info->records = (int)recs.size();
  }
  if (rc != QKX_OK) {
    fclose(f);
    return rc;
  }
  // stream: file -> pinned[k] -> raw device bytes; then swap into the AoS links
  unsigned char* pin[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  void* raw = nullptr;
  double* aos = nullptr;
  const size_t bytes = bin->bytes;
  if (cudaHostAlloc((void**)&pin[0], LIME_CHUNK, cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void**)&pin[1], LIME_CHUNK, cudaHostAllocDefault) != cudaSuccess ||
      cudaMallocAsync(&raw, bytes, c->st) != cudaSuccess ||
      cudaMallocAsync((void**)&aos, sizeof(double) * nwords, c->st) != cudaSuccess) {
    set_error("LIME read: allocation failed");
    rc = QKX_ERR_NOMEM;
  }
  if (rc == QKX_OK && (cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming) != cudaSuccess ||
                       cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming) != cudaSuccess))
    rc = QKX_ERR_CUDA;
  if (rc == QKX_OK && fseeko(f, (off_t)bin->offset, SEEK_SET) != 0) rc = bad("cannot seek to the binary data%s");
  for (size_t off = 0, k = 0; off < bytes && rc == QKX_OK; off += LIME_CHUNK, k ^= 1) {
    const size_t n = std::min(LIME_CHUNK, bytes - off);
    if (cudaEventSynchronize(done[k]) != cudaSuccess) rc = QKX_ERR_CUDA;  // the copy out of pin[k] finished
    if (rc == QKX_OK && fread(pin[k], 1, n, f) != n) rc = bad("short read of the binary data%s");
    if (rc == QKX_OK && cudaMemcpyAsync((unsigned char*)raw + off, pin[k], n, cudaMemcpyHostToDevice, c->st) != cudaSuccess)
      rc = QKX_ERR_CUDA;
    if (rc == QKX_OK && cudaEventRecord(done[k], c->st) != cudaSuccess) rc = QKX_ERR_CUDA;
  }
  fclose(f);
  if (rc == QKX_OK) {
    if (precision == 64)
      k_bswap64<<<swap_grid(nwords), 256, 0, c->st>>>((const unsigned long long*)raw, aos, nwords);
    else
      k_bswap32<<<swap_grid(nwords), 256, 0, c->st>>>((const unsigned*)raw, aos, nwords);
    counted(c);
    const int tsign = (bc_mode == QKX_LINKS_APPLY_BC && c->p.boundaryT == -1) ? -1 : 1;
    k_gauge_aos_to_eo<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>((const double2*)aos, c->U18, c->geom, tsign);
    counted(c);
    if (cudaGetLastError() != cudaSuccess) rc = QKX_ERR_CUDA;
    if (rc == QKX_OK && U_host &&
        cudaMemcpyAsync(U_host, aos, sizeof(double) * nwords, cudaMemcpyDeviceToHost, c->st) != cudaSuccess)
      rc = QKX_ERR_CUDA;
  }
  cudaStreamSynchronize(c->st);
  for (int k = 0; k < 2; k++) {
    if (done[k]) cudaEventDestroy(done[k]);
    if (pin[k]) cudaFreeHost(pin[k]);
  }
  if (raw) cudaFreeAsync(raw, c->st);
  if (aos) cudaFreeAsync(aos, c->st);
  if (rc == QKX_ERR_CUDA) set_error("LIME read: %s", cudaGetErrorString(cudaGetLastError()));
  if (rc != QKX_OK) {
    c->have_gauge = 0;  // the operator links may be partly overwritten
    return rc;
  }
  return gauge_finish(c);
}

int qkx_write_gauge_lime(qkx_ctx* c, const char* path, const double* U_host, const char* message) {
  if (!c || !path) return bad("invalid argument: NULL argument%s");
  if (!U_host && !c->have_gauge) {
    set_error("no gauge field to write");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  const size_t nwords = (size_t)72 * c->V;
  const size_t bytes = nwords * 8;
  double* aos = nullptr;
  unsigned long long* be = nullptr;
  std::vector<unsigned char> host(bytes);
  // every step runs only if the ones before it succeeded; both buffers are freed on every path
  cudaError_t e = cudaMallocAsync((void**)&aos, bytes, c->st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&be, bytes, c->st);
  if (e == cudaSuccess) {
    if (U_host) {
      e = cudaMemcpyAsync(aos, U_host, bytes, cudaMemcpyHostToDevice, c->st);
    } else {
      k_gauge_eo_to_aos<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(c->U18, (double2*)aos, c->geom);
      counted(c);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) {
    // native -> big-endian: the same byte reversal
    k_bswap64<<<swap_grid(nwords), 256, 0, c->st>>>((const unsigned long long*)aos, (double*)be, nwords);
    counted(c);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), be, bytes, cudaMemcpyDeviceToHost, c->st);
  if (aos) cudaFreeAsync(aos, c->st);
  if (be) cudaFreeAsync(be, c->st);
  const cudaError_t es = cudaStreamSynchronize(c->st);
  if (e == cudaSuccess) e = es;
  if (e != cudaSuccess) {
    set_error("LIME write: %s", cudaGetErrorString(e));
    return QKX_ERR_CUDA;
  }

  // the ildg-format text of lib/write_conf_lime.cpp:84 character for character, so that the
  // file is the reference writer's byte for byte
  char xml[1024];
  snprintf(xml, sizeof xml,
           "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n<ildgFormat xmlns=\"http://www.lqkxTM.org/ildg\"\n"
           "            xmlns:xsi=\"http://www.w3.org/2001/XMLSchema-instance\"\n"
           "            xsi:schemaLocation=\"http://www.lqkxTM.org/ildg filefmt.xsd\">\n"
           "  <version> 1.0 </version>\n  <field> su3gauge </field>\n  <precision> 64 </precision>\n"
           "  <lx> %d </lx>\n  <ly> %d </ly>\n  <lz> %d </lz>\n  <lt> %d </lt>\n</ildgFormat>",
           c->p.L[0], c->p.L[1], c->p.L[2], c->p.L[3]);
  const std::string msg = message ? message : "";
  FILE* f = fopen(path, "wb");
  if (!f) return bad("cannot open '%s' for writing", path);
  auto record = [&](const char* type, const void* data, uint64_t n, bool mb, bool me) -> bool {
    unsigned char h[LIME_HDR];
    memset(h, 0, sizeof h);
    h[0] = 0x45, h[1] = 0x67, h[2] = 0x89, h[3] = 0xab;
    h[5] = 1;  // version
    h[6] = (unsigned char)((mb ? 0x80 : 0) | (me ? 0x40 : 0));
    put_be64(h + 8, n);
    strncpy((char*)h + 16, type, 127);
    if (fwrite(h, 1, LIME_HDR, f) != LIME_HDR) return false;
    if (n && fwrite(data, 1, n, f) != n) return false;
    static const unsigned char zeros[8] = {0};
    const size_t pad = (size_t)((8 - (n & 7)) & 7);
    return pad == 0 || fwrite(zeros, 1, pad, f) == pad;
  };
  bool ok = record("ildg-format", xml, strlen(xml), true, false) &&
            record("xlf-info", msg.data(), msg.size(), false, false) &&
            record("ildg-binary-data", host.data(), bytes, false, true);
  ok = (fclose(f) == 0) && ok;
  if (!ok) return bad("write to '%s' failed", path);
  return QKX_OK;
}

}  // extern "C"
