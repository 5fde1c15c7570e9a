// Checkpoints: the save/load that config.cpp:75-262 sketches and leaves
// commented out (parameters, the per-cell grid, GA, SUM and V, the channel
// flags and the kernels), as a versioned binary file.
//
// Layout (little-endian):
//   "LENIACKP"                      8-byte magic
//   u32 version (1), u32 flags (bit 0: a mass-target record follows the
//     fields)
//   u32 n_desc_words, then the LeniaWorldDesc fields in declaration order as
//     32-bit words (ints as i32, floats as IEEE-754 binary32)
//   u32 n_kernels, then per kernel radius, beta_size, b[12], r_a, m, s, h,
//     c0, c1 as 32-bit words
//   u64 step (caller's counter)
//   u32 n_fields, then per field: u32 LeniaField id, u64 float count, the
//     floats (A, V, GA, SUM: everything that carries over between steps)
//   flags bit 0: u32 n_channels, then per channel the conserve_mass target
//     total as an IEEE-754 binary64 (the totals every later step restores;
//     without them a resumed world would take its restored grid's rounded
//     totals as the target and drift from the run that never stopped)
//   u32 CRC-32 (IEEE 802.3 polynomial, reflected) of every byte before it
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "lenia_internal.h"

namespace {

constexpr char kMagic[8] = {'L', 'E', 'N', 'I', 'A', 'C', 'K', 'P'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kFlagMassTarget = 1;

uint32_t crc32_update(uint32_t crc, const unsigned char *p, size_t n)
{
    static uint32_t table[256];
    static bool ready = false;
    if (!ready) {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t c = i;
            for (int k = 0; k < 8; k++) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        ready = true;
    }
    crc = ~crc;
    for (size_t i = 0; i < n; i++) crc = table[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
    return ~crc;
}

struct Writer {
    std::vector<unsigned char> buf;
    void bytes(const void *p, size_t n)
    {
        const unsigned char *c = (const unsigned char *)p;
        buf.insert(buf.end(), c, c + n);
    }
    void u32(uint32_t v) { for (int i = 0; i < 4; i++) buf.push_back((unsigned char)(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; i++) buf.push_back((unsigned char)(v >> (8 * i))); }
    void f32(float f)
    {
        uint32_t v;
        memcpy(&v, &f, 4);
        u32(v);
    }
    void f64(double f)
    {
        uint64_t v;
        memcpy(&v, &f, 8);
        u64(v);
    }
};

struct Reader {
    const std::vector<unsigned char> &buf;
    size_t pos = 0;
    bool ok = true;
    explicit Reader(const std::vector<unsigned char> &b) : buf(b) {}
    bool need(size_t n)
    {
        if (pos + n > buf.size()) ok = false;
        return ok;
    }
    uint32_t u32()
    {
        if (!need(4)) return 0;
        uint32_t v = 0;
        for (int i = 0; i < 4; i++) v |= (uint32_t)buf[pos + i] << (8 * i);
        pos += 4;
        return v;
    }
    uint64_t u64()
    {
        if (!need(8)) return 0;
        uint64_t v = 0;
        for (int i = 0; i < 8; i++) v |= (uint64_t)buf[pos + i] << (8 * i);
        pos += 8;
        return v;
    }
    float f32()
    {
        const uint32_t v = u32();
        float f;
        memcpy(&f, &v, 4);
        return f;
    }
    double f64()
    {
        const uint64_t v = u64();
        double f;
        memcpy(&f, &v, 8);
        return f;
    }
};

// LeniaWorldDesc as 32-bit words in declaration order (every member is a
// 32-bit int or float).
static_assert(sizeof(LeniaWorldDesc) % 4 == 0, "LeniaWorldDesc packs into 32-bit words");
constexpr uint32_t kDescWords = sizeof(LeniaWorldDesc) / 4;

const int kSavedFields[] = {LENIA_FIELD_A, LENIA_FIELD_V, LENIA_FIELD_GA, LENIA_FIELD_SUM};

}  // namespace

extern "C" {

lenia_status lenia_save(lenia_world *w, const LeniaWorldDesc *desc, const LeniaKernelParams *kernels, int n_kernels,
                        unsigned long long step, const char *path)
{
    if (!w || !desc || (n_kernels > 0 && !kernels) || n_kernels < 0 || !path) return LENIA_ERR_INVALID_ARG;
    double target[LENIA_MAX_CHANNELS];
    const int n_target = desc->conserve_mass ? lenia::mass_target_get(w, target, LENIA_MAX_CHANNELS) : 0;
    Writer wr;
    wr.bytes(kMagic, 8);
    wr.u32(kVersion);
    wr.u32(n_target > 0 ? kFlagMassTarget : 0);
    wr.u32(kDescWords);
    uint32_t words[kDescWords];
    memcpy(words, desc, sizeof(LeniaWorldDesc));
    for (uint32_t i = 0; i < kDescWords; i++) wr.u32(words[i]);
    wr.u32((uint32_t)n_kernels);
    for (int k = 0; k < n_kernels; k++) {
        const LeniaKernelParams &p = kernels[k];
        wr.u32((uint32_t)p.radius);
        wr.u32((uint32_t)p.beta_size);
        for (int j = 0; j < LENIA_MAX_BETA; j++) wr.f32(p.b[j]);
        wr.f32(p.r_a);
        wr.f32(p.m);
        wr.f32(p.s);
        wr.f32(p.h);
        wr.u32((uint32_t)p.c0);
        wr.u32((uint32_t)p.c1);
    }
    wr.u64(step);
    wr.u32((uint32_t)(sizeof(kSavedFields) / sizeof(int)));
    std::vector<float> tmp;
    for (int field : kSavedFields) {
        const size_t n = lenia_field_size(w, field);
        tmp.resize(n);
        const lenia_status s = lenia_get_field(w, field, tmp.data(), n, 0);
        if (s != LENIA_OK) return s;
        wr.u32((uint32_t)field);
        wr.u64(n);
        for (size_t i = 0; i < n; i++) wr.f32(tmp[i]);
    }
    if (n_target > 0) {
        wr.u32((uint32_t)n_target);
        for (int c = 0; c < n_target; c++) wr.f64(target[c]);
    }
    wr.u32(crc32_update(0, wr.buf.data(), wr.buf.size()));
    FILE *f = fopen(path, "wb");
    if (!f) return LENIA_ERR_INVALID_ARG;
    const size_t put = fwrite(wr.buf.data(), 1, wr.buf.size(), f);
    const int closed = fclose(f);
    return (put == wr.buf.size() && closed == 0) ? LENIA_OK : LENIA_ERR_INVALID_ARG;
}

lenia_status lenia_load(const char *path, lenia_world **out, unsigned long long *step)
{
    if (!path || !out) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) return LENIA_ERR_INVALID_ARG;
    std::vector<unsigned char> buf;
    unsigned char chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    fclose(f);
    if (buf.size() < 8 + 4 || memcmp(buf.data(), kMagic, 8) != 0) {
        fprintf(stderr, "lenia_load: %s is not a checkpoint\n", path);
        return LENIA_ERR_INVALID_ARG;
    }
    const size_t body = buf.size() - 4;
    uint32_t stored = 0;
    for (int i = 0; i < 4; i++) stored |= (uint32_t)buf[body + i] << (8 * i);
    if (crc32_update(0, buf.data(), body) != stored) {
        fprintf(stderr, "lenia_load: %s fails its checksum\n", path);
        return LENIA_ERR_INVALID_ARG;
    }
    Reader rd(buf);
    rd.pos = 8;
    const uint32_t version = rd.u32();
    const uint32_t flags = rd.u32();
    if (version != kVersion) {
        fprintf(stderr, "lenia_load: %s has version %u, this library reads %u\n", path, version, kVersion);
        return LENIA_ERR_UNSUPPORTED;
    }
    // a descriptor written before trailing fields were added is read with
    // those fields 0 (their reference behaviour)
    const uint32_t nwords = rd.u32();
    if (nwords > kDescWords || nwords < 2) return LENIA_ERR_UNSUPPORTED;
    uint32_t words[kDescWords] = {};
    for (uint32_t i = 0; i < nwords; i++) words[i] = rd.u32();
    LeniaWorldDesc desc;
    memcpy(&desc, words, sizeof(desc));
    const uint32_t nk = rd.u32();
    if (!rd.ok || nk > LENIA_MAX_KERNELS) return LENIA_ERR_INVALID_ARG;
    std::vector<LeniaKernelParams> ks(nk);
    for (uint32_t k = 0; k < nk; k++) {
        LeniaKernelParams &p = ks[k];
        p.radius = (int)rd.u32();
        p.beta_size = (int)rd.u32();
        for (int j = 0; j < LENIA_MAX_BETA; j++) p.b[j] = rd.f32();
        p.r_a = rd.f32();
        p.m = rd.f32();
        p.s = rd.f32();
        p.h = rd.f32();
        p.c0 = (int)rd.u32();
        p.c1 = (int)rd.u32();
    }
    const uint64_t st = rd.u64();
    const uint32_t nf = rd.u32();
    if (!rd.ok) return LENIA_ERR_INVALID_ARG;
    lenia_world *w = nullptr;
    lenia_status s = lenia_create(&desc, ks.data(), (int)nk, &w);
    if (s != LENIA_OK) return s;
    std::vector<float> tmp;
    for (uint32_t i = 0; i < nf && s == LENIA_OK; i++) {
        const int field = (int)rd.u32();
        const uint64_t n = rd.u64();
        if (!rd.ok || !rd.need(4 * n) || n != lenia_field_size(w, field)) {
            s = LENIA_ERR_INVALID_ARG;
            break;
        }
        tmp.resize(n);
        for (uint64_t j = 0; j < n; j++) tmp[j] = rd.f32();
        s = lenia_set_field(w, field, tmp.data(), n, 0);
    }
    // the saved conserve_mass totals replace the ones lenia_set_field just
    // recorded from the restored grid
    if (s == LENIA_OK && (flags & kFlagMassTarget)) {
        const uint32_t nc = rd.u32();
        double target[LENIA_MAX_CHANNELS];
        if (!rd.ok || nc > LENIA_MAX_CHANNELS || nc != (uint32_t)desc.channels) s = LENIA_ERR_INVALID_ARG;
        for (uint32_t c = 0; c < nc && s == LENIA_OK; c++) target[c] = rd.f64();
        if (s == LENIA_OK && !rd.ok) s = LENIA_ERR_INVALID_ARG;
        if (s == LENIA_OK && desc.conserve_mass) s = lenia::mass_target_set(w, target, (int)nc);
    }
    if (s != LENIA_OK) {
        lenia_destroy(w);
        return s;
    }
    if (step) *step = st;
    *out = w;
    return LENIA_OK;
}

}  // extern "C"
