// ix_radiance_host.cpp -- the radiance frame codec (include/ix_radiance.h): the byte shuffle,
// an LZ4 block compressor / bounded decompressor, the payload encoder and the bounded
// decoder of crates/indicatrix-net/src/radiance/, and the host side of the device forms
// (kernels in ix_radiance.cu).
//
// The LZ4 block format (sequences of a token, literal run, 16-bit offset and match run;
// the block ends with a literal-only sequence; the last 5 bytes are literals and no match
// starts within the last 12) is the published format lz4_flex 0.14.0 reads and writes.
// The compressor here is a greedy single-probe hash matcher of its own; any valid block
// decodes to the same bytes, so only the format has to agree.

#include "../../include/ix_radiance.h"
#include "ix_backend_state.h"

#include <cmath>
#include <cstring>
#include <vector>

using namespace ixh;

namespace ix {
namespace rad {
cudaError_t launch_encode(const double* sums, uint64_t values, int shuffle, uint8_t* out, cudaStream_t s);
cudaError_t launch_decode_add(const uint8_t* payload, uint64_t pixels, int shuffled, float* acc,
                              unsigned int* dropped, cudaStream_t s);
}  // namespace rad
}  // namespace ix

struct RadianceState {
    uint8_t* d_payload = nullptr;  // encoded / decoded bytes on the device
    size_t payload_cap = 0;
    unsigned int* d_dropped = nullptr;
    uint8_t* h_bytes = nullptr;    // pinned host copy of the same bytes
    size_t hbytes_cap = 0;
};

void radiance_state_free(RadianceState* r) {
    if (!r) return;
    cudaFree(r->d_payload);
    cudaFree(r->d_dropped);
    if (r->h_bytes) cudaFreeHost(r->h_bytes);
    delete r;
}

namespace {

constexpr size_t PLANES = 4;
constexpr size_t MIN_MATCH = 4;
constexpr size_t LAST_LITERALS = 5;
constexpr size_t MF_LIMIT = 12;
constexpr int HASH_BITS = 16;

inline uint32_t read32(const uint8_t* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
inline uint32_t hash4(uint32_t v) { return (v * 2654435761u) >> (32 - HASH_BITS); }

// Writes one sequence; false when it does not fit in `cap`.
bool put_sequence(uint8_t* dst, size_t cap, size_t* op, const uint8_t* lit, size_t lit_len, size_t offset,
                  size_t match_len, bool last) {
    size_t o = *op;
    auto put = [&](uint8_t v) {
        if (o >= cap) return false;
        dst[o++] = v;
        return true;
    };
    const size_t ml = last ? 0 : match_len - MIN_MATCH;
    const uint8_t token = (uint8_t)((std::min<size_t>(lit_len, 15) << 4) | (last ? 0 : std::min<size_t>(ml, 15)));
    if (!put(token)) return false;
    if (lit_len >= 15) {
        size_t r = lit_len - 15;
        for (; r >= 255; r -= 255)
            if (!put(255)) return false;
        if (!put((uint8_t)r)) return false;
    }
    if (lit_len > cap - o) return false;
    std::memcpy(dst + o, lit, lit_len);
    o += lit_len;
    if (!last) {
        if (!put((uint8_t)(offset & 0xFF)) || !put((uint8_t)(offset >> 8))) return false;
        if (ml >= 15) {
            size_t r = ml - 15;
            for (; r >= 255; r -= 255)
                if (!put(255)) return false;
            if (!put((uint8_t)r)) return false;
        }
    }
    *op = o;
    return true;
}

// One LZ4 block of src[0, n) into dst; returns the block's length, or 0 when it does not
// fit in `cap` (an n of 0 gives the one-byte empty block).
size_t lz4_compress(const uint8_t* src, size_t n, uint8_t* dst, size_t cap) {
    size_t op = 0, anchor = 0;
    if (n >= MF_LIMIT + 1) {
        std::vector<uint32_t> table((size_t)1 << HASH_BITS, UINT32_MAX);
        const size_t last_start = n - MF_LIMIT;     // a match starts at or before this
        const size_t match_end = n - LAST_LITERALS;  // and ends at or before this
        size_t ip = 0;
        while (ip <= last_start) {
            const uint32_t seq = read32(src + ip);
            const uint32_t h = hash4(seq);
            const uint32_t ref = table[h];
            table[h] = (uint32_t)ip;
            if (ref != UINT32_MAX && ip - ref <= 65535 && read32(src + ref) == seq) {
                size_t len = MIN_MATCH;
                while (ip + len < match_end && src[ref + len] == src[ip + len]) ++len;
                if (!put_sequence(dst, cap, &op, src + anchor, ip - anchor, ip - ref, len, false)) return 0;
                ip += len;
                anchor = ip;
                if (ip - 2 <= last_start && ip >= 2) table[hash4(read32(src + ip - 2))] = (uint32_t)(ip - 2);
            } else {
                // Skip faster through incompressible runs.
                ip += 1 + ((ip - anchor) >> 6);
            }
        }
    }
    if (!put_sequence(dst, cap, &op, src + anchor, n - anchor, 0, 0, true)) return 0;
    return op;
}

// Decodes one LZ4 block into at most `cap` bytes; false on a malformed block or one
// whose output would pass `cap` (the bound holds whatever the block claims).
bool lz4_decompress(const uint8_t* src, size_t n, uint8_t* dst, size_t cap, size_t* out_len) {
    size_t ip = 0, op = 0;
    for (;;) {
        if (ip >= n) return false;
        const uint8_t token = src[ip++];
        size_t lit = token >> 4;
        if (lit == 15) {
            uint8_t b;
            do {
                if (ip >= n) return false;
                b = src[ip++];
                lit += b;
                if (lit > cap) return false;
            } while (b == 255);
        }
        if (lit > n - ip || lit > cap - op) return false;
        std::memcpy(dst + op, src + ip, lit);
        ip += lit;
        op += lit;
        if (ip == n) break;  // the literal-only last sequence
        if (n - ip < 2) return false;
        const size_t off = (size_t)src[ip] | ((size_t)src[ip + 1] << 8);
        ip += 2;
        if (off == 0 || off > op) return false;
        size_t ml = (token & 15u) + MIN_MATCH;
        if ((token & 15u) == 15u) {
            uint8_t b;
            do {
                if (ip >= n) return false;
                b = src[ip++];
                ml += b;
                if (ml > cap) return false;
            } while (b == 255);
        }
        if (ml > cap - op) return false;
        const uint8_t* m = dst + op - off;
        for (size_t k = 0; k < ml; ++k) dst[op + k] = m[k];  // overlapping copies repeat
        op += ml;
    }
    *out_len = op;
    return true;
}

void shuffle_bytes(const uint8_t* src, uint8_t* dst, size_t len) {
    const size_t n = len / PLANES;
    for (size_t i = 0; i < n; ++i)
        for (size_t k = 0; k < PLANES; ++k) dst[k * n + i] = src[PLANES * i + k];
}
void unshuffle_bytes(const uint8_t* src, uint8_t* dst, size_t len) {
    const size_t n = len / PLANES;
    for (size_t i = 0; i < n; ++i)
        for (size_t k = 0; k < PLANES; ++k) dst[PLANES * i + k] = src[k * n + i];
}

// is_valid_sample (shuffle.rs:23): every component finite and not negative.
inline bool valid_sample(const float v[3]) {
    return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]) && v[0] >= 0.0f && v[1] >= 0.0f &&
           v[2] >= 0.0f;
}

// PayloadDecoder::prepare (payload.rs:264-301): the bounded-decode checks in order, then
// the raw bytes (`*raw`) or the decompressed planes (`planes`, which must hold raw_len).
int prepare(uint32_t encoding, uint32_t raw_len, const uint8_t* wire, size_t wire_len, uint32_t width,
            uint32_t height, std::vector<uint8_t>* planes, uint8_t* planes_buf, const uint8_t** raw,
            bool* shuffled) {
    const uint64_t expected = (uint64_t)width * height * IX_RADIANCE_BYTES_PER_PIXEL;
    if (expected > IX_MAX_FRAME_LEN) return IX_RADIANCE_TOO_LARGE;
    if ((uint64_t)raw_len != expected) return IX_RADIANCE_RAW_LEN_MISMATCH;
    *shuffled = false;
    if (encoding == IX_PAYLOAD_RAW) {
        // decode_borrowed (radiance/mod.rs:212): the length must match exactly.
        if ((uint64_t)wire_len != expected || (!wire && wire_len)) return IX_RADIANCE_LENGTH_MISMATCH;
        *raw = wire;
        return IX_RADIANCE_OK;
    }
    if (!ix_payload_encoding_supported(encoding)) return IX_RADIANCE_UNSUPPORTED_ENCODING;
    if (expected == 0) {
        *raw = wire;
        return IX_RADIANCE_OK;
    }
    uint8_t* out = planes_buf;
    if (!out) {
        planes->resize((size_t)expected);
        out = planes->data();
    }
    size_t got = 0;
    if (!wire || !lz4_decompress(wire, wire_len, out, (size_t)expected, &got)) return IX_RADIANCE_DECOMPRESS_FAILED;
    if (got != expected) return IX_RADIANCE_SHORT_OUTPUT;
    *raw = out;
    *shuffled = true;
    return IX_RADIANCE_OK;
}

RadianceState* rstate(ix_backend* b) {
    if (!b->radiance) b->radiance = new RadianceState();
    return b->radiance;
}

}  // namespace

extern "C" {

int ix_payload_encoding_supported(uint32_t encoding) {
    return encoding == IX_PAYLOAD_RAW || encoding == IX_PAYLOAD_SHUFFLE_LZ4;
}

size_t ix_payload_max_encoded_len(size_t raw_len) { return raw_len + raw_len / 255 + 16; }

int ix_radiance_shuffle(const uint8_t* src, uint8_t* dst, size_t len) {
    if (len % PLANES != 0 || (len && (!src || !dst))) return IX_RADIANCE_LENGTH_MISMATCH;
    shuffle_bytes(src, dst, len);
    return IX_RADIANCE_OK;
}

int ix_radiance_unshuffle(const uint8_t* src, uint8_t* dst, size_t len) {
    if (len % PLANES != 0 || (len && (!src || !dst))) return IX_RADIANCE_LENGTH_MISMATCH;
    unshuffle_bytes(src, dst, len);
    return IX_RADIANCE_OK;
}

int ix_payload_encode(uint32_t encoding, const uint8_t* raw, size_t raw_len, uint8_t* wire, size_t wire_cap,
                      size_t* wire_len, uint32_t* used_encoding) {
    if (!wire_len || !used_encoding || (raw_len && !raw)) return IX_RADIANCE_LENGTH_MISMATCH;
    // PayloadEncoder::new: an encoding this build cannot handle becomes Raw.
    if (!ix_payload_encoding_supported(encoding)) encoding = IX_PAYLOAD_RAW;
    if (encoding == IX_PAYLOAD_SHUFFLE_LZ4 && raw_len > 0 && raw_len % PLANES == 0 && wire) {
        std::vector<uint8_t> planes(raw_len);
        shuffle_bytes(raw, planes.data(), raw_len);
        // Only a block smaller than the raw bytes is sent compressed (payload.rs:152).
        const size_t cap = std::min(wire_cap, raw_len - 1);
        const size_t len = cap ? lz4_compress(planes.data(), raw_len, wire, cap) : 0;
        if (len > 0 && len < raw_len) {
            *wire_len = len;
            *used_encoding = IX_PAYLOAD_SHUFFLE_LZ4;
            return IX_RADIANCE_OK;
        }
    }
    if (wire_cap < raw_len || (raw_len && !wire)) return IX_RADIANCE_BUFFER_TOO_SMALL;
    if (raw_len) std::memcpy(wire, raw, raw_len);
    *wire_len = raw_len;
    *used_encoding = IX_PAYLOAD_RAW;
    return IX_RADIANCE_OK;
}

int ix_payload_decode_and_add(uint32_t encoding, uint32_t raw_len, const uint8_t* wire, size_t wire_len,
                              uint32_t width, uint32_t height, float* acc, uint32_t* dropped) {
    const uint64_t pixels = (uint64_t)width * height;
    if (pixels && !acc) return IX_RADIANCE_LENGTH_MISMATCH;
    std::vector<uint8_t> planes;
    const uint8_t* bytes = nullptr;
    bool shuffled = false;
    const int rc = prepare(encoding, raw_len, wire, wire_len, width, height, &planes, nullptr, &bytes, &shuffled);
    if (rc != IX_RADIANCE_OK) return rc;
    const size_t n = (size_t)pixels * 3;
    uint32_t drop = 0;
    for (uint64_t p = 0; p < pixels; ++p) {
        float v[3];
        for (int c = 0; c < 3; ++c) {
            const size_t i = (size_t)p * 3 + c;
            uint8_t b4[4];
            for (size_t k = 0; k < PLANES; ++k) b4[k] = shuffled ? bytes[k * n + i] : bytes[PLANES * i + k];
            std::memcpy(&v[c], b4, 4);
        }
        if (valid_sample(v)) {
            for (int c = 0; c < 3; ++c) acc[3 * p + c] += v[c];
        } else if (drop != UINT32_MAX) {
            ++drop;
        }
    }
    if (dropped) *dropped = drop;
    return IX_RADIANCE_OK;
}

int ix_payload_decode(uint32_t encoding, uint32_t raw_len, const uint8_t* wire, size_t wire_len, uint32_t width,
                      uint32_t height, float* out) {
    const uint64_t pixels = (uint64_t)width * height;
    if (pixels && !out) return IX_RADIANCE_LENGTH_MISMATCH;
    std::vector<uint8_t> planes;
    const uint8_t* bytes = nullptr;
    bool shuffled = false;
    const int rc = prepare(encoding, raw_len, wire, wire_len, width, height, &planes, nullptr, &bytes, &shuffled);
    if (rc != IX_RADIANCE_OK) return rc;
    const size_t len = (size_t)pixels * IX_RADIANCE_BYTES_PER_PIXEL;
    if (shuffled)
        unshuffle_bytes(bytes, (uint8_t*)out, len);
    else if (len)
        std::memcpy(out, bytes, len);
    return IX_RADIANCE_OK;
}

int ix_payload_encode_device(ix_backend* b, uint32_t encoding, const double* d_sums, uint32_t width, uint32_t height,
                             uint8_t* wire, size_t wire_cap, size_t* wire_len, uint32_t* used_encoding,
                             void* stream) {
    if (!b || b->lost) return IX_RADIANCE_DECLINED;
    if (!wire_len || !used_encoding) return IX_RADIANCE_LENGTH_MISMATCH;
    const uint64_t raw_len = (uint64_t)width * height * IX_RADIANCE_BYTES_PER_PIXEL;
    if (raw_len > IX_MAX_FRAME_LEN) return IX_RADIANCE_TOO_LARGE;
    if (!ix_payload_encoding_supported(encoding)) encoding = IX_PAYLOAD_RAW;
    if (raw_len == 0) {
        *wire_len = 0;
        *used_encoding = encoding == IX_PAYLOAD_SHUFFLE_LZ4 ? IX_PAYLOAD_RAW : encoding;
        return IX_RADIANCE_OK;
    }
    if (!d_sums || !wire) return IX_RADIANCE_LENGTH_MISMATCH;
    Turn turn(b);
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_RADIANCE_DECLINED;
    const cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    RadianceState* r = rstate(b);
    cudaError_t e = grow_device(&r->d_payload, &r->payload_cap, (size_t)raw_len);
    if (e == cudaSuccess) e = grow_pinned(&r->h_bytes, &r->hbytes_cap, (size_t)raw_len);
    if (fail(b, e, "payload buffers")) return IX_RADIANCE_DECLINED;
    const bool lz4 = encoding == IX_PAYLOAD_SHUFFLE_LZ4;
    e = ix::rad::launch_encode(d_sums, raw_len / 4, lz4 ? 1 : 0, r->d_payload, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r->h_bytes, r->d_payload, (size_t)raw_len, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (fail(b, e, "payload encode")) return IX_RADIANCE_DECLINED;
    if (lz4) {
        const size_t cap = std::min<size_t>(wire_cap, (size_t)raw_len - 1);
        const size_t len = cap ? lz4_compress(r->h_bytes, (size_t)raw_len, wire, cap) : 0;
        if (len > 0 && len < raw_len) {
            *wire_len = len;
            *used_encoding = IX_PAYLOAD_SHUFFLE_LZ4;
            return IX_RADIANCE_OK;
        }
        // Not smaller: the raw bytes, as the encoder's fallback sends them.
        if (wire_cap < raw_len) return IX_RADIANCE_BUFFER_TOO_SMALL;
        unshuffle_bytes(r->h_bytes, wire, (size_t)raw_len);
    } else {
        if (wire_cap < raw_len) return IX_RADIANCE_BUFFER_TOO_SMALL;
        std::memcpy(wire, r->h_bytes, (size_t)raw_len);
    }
    *wire_len = (size_t)raw_len;
    *used_encoding = IX_PAYLOAD_RAW;
    return IX_RADIANCE_OK;
}

int ix_payload_decode_and_add_device(ix_backend* b, uint32_t encoding, uint32_t raw_len, const uint8_t* wire,
                                     size_t wire_len, uint32_t width, uint32_t height, float* d_acc,
                                     uint32_t* dropped, void* stream) {
    if (!b || b->lost) return IX_RADIANCE_DECLINED;
    const uint64_t pixels = (uint64_t)width * height;
    if (pixels && !d_acc) return IX_RADIANCE_LENGTH_MISMATCH;
    const uint64_t expected = pixels * IX_RADIANCE_BYTES_PER_PIXEL;
    Turn turn(b);
    RadianceState* r = rstate(b);
    // The checks and the decompression run on the host, into the pinned buffer.
    if (expected <= IX_MAX_FRAME_LEN &&
        fail(b, grow_pinned(&r->h_bytes, &r->hbytes_cap, std::max<size_t>((size_t)expected, 1)), "payload host"))
        return IX_RADIANCE_DECLINED;
    std::vector<uint8_t> unused;
    const uint8_t* bytes = nullptr;
    bool shuffled = false;
    const int rc =
        prepare(encoding, raw_len, wire, wire_len, width, height, &unused, r->h_bytes, &bytes, &shuffled);
    if (rc != IX_RADIANCE_OK) return rc;
    if (dropped) *dropped = 0;
    if (pixels == 0) return IX_RADIANCE_OK;
    if (fail(b, cudaSetDevice(b->device), "set device")) return IX_RADIANCE_DECLINED;
    const cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
    cudaError_t e = grow_device(&r->d_payload, &r->payload_cap, (size_t)expected);
    if (e == cudaSuccess && !r->d_dropped) e = cudaMalloc((void**)&r->d_dropped, sizeof(unsigned int));
    if (fail(b, e, "payload buffers")) return IX_RADIANCE_DECLINED;
    if (bytes != r->h_bytes) std::memcpy(r->h_bytes, bytes, (size_t)expected);  // raw: stage the caller's bytes
    e = cudaMemcpyAsync(r->d_payload, r->h_bytes, (size_t)expected, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(r->d_dropped, 0, sizeof(unsigned int), st);
    if (e == cudaSuccess) e = ix::rad::launch_decode_add(r->d_payload, pixels, shuffled ? 1 : 0, d_acc, r->d_dropped, st);
    unsigned int h_drop = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_drop, r->d_dropped, sizeof(h_drop), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (fail(b, e, "payload decode")) return IX_RADIANCE_DECLINED;
    if (dropped) *dropped = h_drop;
    return IX_RADIANCE_OK;
}

}  // extern "C"
