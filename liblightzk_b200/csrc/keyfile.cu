// keyfile.cu -- proving keys on disk: lzk_pk_save, lzk_pk_load, lzk_pk_free.
//
// The reference regenerates its proving key on every run from unseeded
// randomness (Groth16::Setup, include/protocol/groth16.cuh:48-152) and
// keeps it only in memory; a prover service instead loads each circuit's
// key once, builds its resident tables from it and drops the file's copy.
// The file holds exactly what lzk_prover_create reads: the five query
// arrays and alpha, beta, delta, plus the circuit shape they belong to.
//
// Layout (little-endian, version 1):
//   header, 128 bytes:
//     0   char[8]  magic "LZKG16PK"
//     8   u32      version (1)
//     12  u32      header bytes (128)
//     16  u64      n_vars
//     24  u64      n_public
//     32  u32      log_domain
//     36  u32      reserved (0)
//     40  u64[5]   points in a, b1, b2, l, h (n_vars, n_vars, n_vars,
//                  n_vars - n_public - 1, 2^log_domain - 1)
//     80  u64      checksum of the body (below)
//     88  ...      zero up to 128
//   body: alpha1, beta1, delta1 (G1 affine, 64 B each), beta2, delta2 (G2
//   affine, 128 B each), then the a, b1 (G1), b2 (G2), l, h (G1) arrays.
// Coordinates are the Montgomery-form limbs of include/lzk.h, as the arrays
// sit in device memory.  The checksum folds the body as 64-bit words:
// h = (h xor w) * 0x100000001b3, rotated left by 29 after every word,
// from h = 0xcbf29ce484222325 (a word-wise FNV-1a variant).
#include "common.cuh"
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

struct lzk_pk {
    void* dev = nullptr;    // one device allocation holding the five arrays
    size_t bytes = 0;
};

namespace lzk {

constexpr char kMagic[8] = {'L', 'Z', 'K', 'G', '1', '6', 'P', 'K'};
constexpr uint32_t kVersion = 1, kHeader = 128;

struct KeyHeader {
    char magic[8];
    uint32_t version, header_bytes;
    uint64_t n_vars, n_public;
    uint32_t log_domain, reserved;
    uint64_t count[5];
    uint64_t checksum;
    uint8_t pad[kHeader - 88];
};
static_assert(sizeof(KeyHeader) == kHeader, "key file header is 128 bytes");

struct Checksum {
    uint64_t h = 0xcbf29ce484222325ull;
    void feed(const void* p, size_t n)   // n a multiple of 8
    {
        const uint64_t* w = static_cast<const uint64_t*>(p);
        for (size_t i = 0; i < n / 8; i++) {
            h = (h ^ w[i]) * 0x100000001b3ull;
            h = (h << 29) | (h >> 35);
        }
    }
};

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() { if (f) std::fclose(f); }
};

constexpr size_t kG1 = sizeof(lzk_g1_affine_t), kG2 = sizeof(lzk_g2_affine_t);
constexpr size_t kChunk = size_t(64) << 20;   // staging buffer for the copies

static bool expected_counts(uint64_t n_vars, uint64_t n_public, uint32_t log_domain, uint64_t c[5])
{
    if (log_domain < 1 || log_domain > 24 || n_vars < n_public + 1) return false;
    c[0] = c[1] = c[2] = n_vars;
    c[3] = n_vars - n_public - 1;
    c[4] = (uint64_t(1) << log_domain) - 1;
    return true;
}

static size_t array_bytes(int q, uint64_t count) { return count * (q == 2 ? kG2 : kG1); }

}  // namespace lzk

using namespace lzk;

extern "C" {

int lzk_pk_save(const char* path, const lzk_groth16_pk* pk, const lzk_pk_info* info)
{
    if (!path || !pk || !info) return LZK_EINVAL;
    KeyHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.header_bytes = kHeader;
    h.n_vars = info->n_vars;
    h.n_public = info->n_public;
    h.log_domain = info->log_domain;
    if (!expected_counts(h.n_vars, h.n_public, h.log_domain, h.count)) return LZK_EINVAL;
    const void* arr[5] = {pk->a_query, pk->b1_query, pk->b2_query, pk->l_query, pk->h_query};
    for (int q = 0; q < 5; q++)
        if (h.count[q] && !arr[q]) return LZK_EINVAL;
    File f(path, "wb");
    if (!f.f) return LZK_EIO;
    // header first (its checksum is rewritten at the end)
    if (std::fwrite(&h, sizeof(h), 1, f.f) != 1) return LZK_EIO;
    Checksum cs;
    const lzk_g1_affine_t g1[3] = {pk->alpha1, pk->beta1, pk->delta1};
    const lzk_g2_affine_t g2[2] = {pk->beta2, pk->delta2};
    cs.feed(g1, sizeof(g1));
    cs.feed(g2, sizeof(g2));
    if (std::fwrite(g1, sizeof(g1), 1, f.f) != 1 || std::fwrite(g2, sizeof(g2), 1, f.f) != 1) return LZK_EIO;
    void* stage = nullptr;
    LZK_CUDA(cudaMallocHost(&stage, kChunk));
    int rc = LZK_OK;
    for (int q = 0; q < 5 && rc == LZK_OK; q++) {
        size_t total = array_bytes(q, h.count[q]);
        const char* src = static_cast<const char*>(arr[q]);
        for (size_t o = 0; o < total && rc == LZK_OK; o += kChunk) {
            size_t n = total - o < kChunk ? total - o : kChunk;
            cudaError_t e = cudaMemcpy(stage, src + o, n, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) { rc = cuda_status(e); break; }
            cs.feed(stage, n);
            if (std::fwrite(stage, 1, n, f.f) != n) rc = LZK_EIO;
        }
    }
    cudaFreeHost(stage);
    if (rc != LZK_OK) return rc;
    h.checksum = cs.h;
    if (std::fseek(f.f, 0, SEEK_SET) != 0 || std::fwrite(&h, sizeof(h), 1, f.f) != 1) return LZK_EIO;
    if (std::fflush(f.f) != 0) return LZK_EIO;
    return LZK_OK;
}

int lzk_pk_load(const char* path, lzk_pk** out, lzk_groth16_pk* view, lzk_pk_info* info)
{
    if (!path || !out || !view) return LZK_EINVAL;
    *out = nullptr;
    File f(path, "rb");
    if (!f.f) return LZK_EIO;
    KeyHeader h;
    if (std::fread(&h, sizeof(h), 1, f.f) != 1) return LZK_EIO;
    if (std::memcmp(h.magic, kMagic, 8) != 0 || h.version != kVersion || h.header_bytes != kHeader) return LZK_EIO;
    uint64_t want[5];
    if (!expected_counts(h.n_vars, h.n_public, h.log_domain, want)) return LZK_EIO;
    for (int q = 0; q < 5; q++)
        if (h.count[q] != want[q]) return LZK_EIO;
    size_t off[6] = {0};
    for (int q = 0; q < 5; q++) off[q + 1] = off[q] + align_up(array_bytes(q, h.count[q]));
    // the file must be exactly header + constants + arrays
    size_t body = 3 * kG1 + 2 * kG2;
    for (int q = 0; q < 5; q++) body += array_bytes(q, h.count[q]);
    if (std::fseek(f.f, 0, SEEK_END) != 0) return LZK_EIO;
    long end = std::ftell(f.f);
    if (end < 0 || (size_t)end != kHeader + body || std::fseek(f.f, kHeader, SEEK_SET) != 0) return LZK_EIO;
    lzk_g1_affine_t g1[3];
    lzk_g2_affine_t g2[2];
    if (std::fread(g1, sizeof(g1), 1, f.f) != 1 || std::fread(g2, sizeof(g2), 1, f.f) != 1) return LZK_EIO;
    Checksum cs;
    cs.feed(g1, sizeof(g1));
    cs.feed(g2, sizeof(g2));
    lzk_pk* pk = new (std::nothrow) lzk_pk();
    if (!pk) return LZK_ENOMEM;
    pk->bytes = off[5];
    if (dev_malloc(&pk->dev, pk->bytes) != LZK_OK) {
        delete pk;
        return LZK_ENOMEM;
    }
    void* stage = nullptr;
    int rc = cuda_status(cudaMallocHost(&stage, kChunk));
    char* dev = static_cast<char*>(pk->dev);
    for (int q = 0; q < 5 && rc == LZK_OK; q++) {
        size_t total = array_bytes(q, h.count[q]);
        for (size_t o = 0; o < total && rc == LZK_OK; o += kChunk) {
            size_t n = total - o < kChunk ? total - o : kChunk;
            if (std::fread(stage, 1, n, f.f) != n) { rc = LZK_EIO; break; }
            cs.feed(stage, n);
            rc = cuda_status(cudaMemcpy(dev + off[q] + o, stage, n, cudaMemcpyHostToDevice));
        }
    }
    if (stage) cudaFreeHost(stage);
    if (rc == LZK_OK && cs.h != h.checksum) rc = LZK_EIO;
    if (rc != LZK_OK) {
        cudaFree(pk->dev);
        delete pk;
        return rc;
    }
    std::memset(view, 0, sizeof(*view));
    view->a_query = reinterpret_cast<const lzk_g1_affine_t*>(dev + off[0]);
    view->b1_query = reinterpret_cast<const lzk_g1_affine_t*>(dev + off[1]);
    view->b2_query = reinterpret_cast<const lzk_g2_affine_t*>(dev + off[2]);
    view->l_query = reinterpret_cast<const lzk_g1_affine_t*>(dev + off[3]);
    view->h_query = reinterpret_cast<const lzk_g1_affine_t*>(dev + off[4]);
    view->alpha1 = g1[0];
    view->beta1 = g1[1];
    view->delta1 = g1[2];
    view->beta2 = g2[0];
    view->delta2 = g2[1];
    if (info) {
        info->n_vars = h.n_vars;
        info->n_public = h.n_public;
        info->log_domain = h.log_domain;
        info->version = h.version;
    }
    *out = pk;
    return LZK_OK;
}

int lzk_pk_free(lzk_pk* pk)
{
    if (!pk) return LZK_EINVAL;
    if (pk->dev) cudaFree(pk->dev);
    delete pk;
    return LZK_OK;
}

}  // extern "C"
