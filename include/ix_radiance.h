/*
 * ix_radiance.h -- the radiance frame codec of the distributed-render wire protocol, and
 * its device forms for a CUDA lane whose per-pixel sums live in GPU memory.
 *
 * Reference interfaces replaced (crates/indicatrix-net/src/, paths in the project):
 *   radiance/shuffle.rs:35-75        shuffle_into / unshuffle_into   -> ix_radiance_shuffle /
 *                                                                        ix_radiance_unshuffle
 *   radiance/shuffle.rs:23-27        is_valid_sample                 (the add rule below)
 *   radiance/payload.rs:99-160       PayloadEncoder::encode          -> ix_payload_encode
 *   radiance/payload.rs:205-245      PayloadDecoder::decode_and_add  -> ix_payload_decode_and_add
 *   radiance/payload.rs:247-262      PayloadDecoder::decode_to_vec   -> ix_payload_decode
 *   messages/encoding.rs:43-70       PayloadEncoding                 -> IX_PAYLOAD_*
 *   framing/mod.rs:26                MAX_FRAME_LEN                   -> IX_MAX_FRAME_LEN
 *   (this library's own)             ix_payload_encode_device / ix_payload_decode_and_add_device:
 *                                    the same payloads from / into per-pixel sums in device
 *                                    memory, the byte shuffle and the valid-sample add done
 *                                    by kernels.
 *
 * A payload is a frame of Vec3 f32 radiance (12 bytes per pixel, little-endian), Raw or
 * byte-shuffled into 4 planes and compressed as one LZ4 block (the block format of
 * lz4_flex 0.14.0, which the reference links; this file holds its own implementation of
 * the published format).  ShuffleZstd is not supported by this build: the encoder falls
 * back to Raw and the decoder answers IX_RADIANCE_UNSUPPORTED_ENCODING, as a reference
 * build without the `compression` feature does for every compressed encoding.
 */
#ifndef IX_RADIANCE_H
#define IX_RADIANCE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { IX_PAYLOAD_RAW = 0, IX_PAYLOAD_SHUFFLE_ZSTD = 1, IX_PAYLOAD_SHUFFLE_LZ4 = 2 };

/* RadianceError (radiance/mod.rs:68-121) as codes; 0 = Ok. */
enum {
    IX_RADIANCE_OK = 0,
    IX_RADIANCE_LENGTH_MISMATCH = 1,     /* raw bytes != width * height * 12             */
    IX_RADIANCE_TOO_LARGE = 3,           /* width * height * 12 > IX_MAX_FRAME_LEN        */
    IX_RADIANCE_RAW_LEN_MISMATCH = 4,    /* header raw_len != width * height * 12         */
    IX_RADIANCE_UNSUPPORTED_ENCODING = 5,
    IX_RADIANCE_DECOMPRESS_FAILED = 6,   /* corrupt block, or output past raw_len         */
    IX_RADIANCE_SHORT_OUTPUT = 7,        /* block decoded to fewer than raw_len bytes     */
    IX_RADIANCE_BUFFER_TOO_SMALL = 8,    /* caller's wire buffer below the encoded size   */
    IX_RADIANCE_DECLINED = 16            /* device form: backend lost or CUDA error       */
};

#define IX_MAX_FRAME_LEN (512u * 1024u * 1024u)
#define IX_RADIANCE_BYTES_PER_PIXEL 12u

struct ix_backend;

/* Whether this build encodes and decodes `encoding` (PayloadEncoding::is_supported). */
int ix_payload_encoding_supported(uint32_t encoding);

/* Bytes an encoded payload of `raw_len` raw bytes can need (the LZ4 worst case, and at
 * least raw_len for the Raw fallback). */
size_t ix_payload_max_encoded_len(size_t raw_len);

/* The byte shuffle: `len` (a multiple of 4) bytes of little-endian f32 values into 4
 * planes, and back.  Bit-exact for every f32 bit pattern. */
int ix_radiance_shuffle(const uint8_t* src, uint8_t* dst, size_t len);
int ix_radiance_unshuffle(const uint8_t* src, uint8_t* dst, size_t len);

/* PayloadEncoder::encode: shuffle + LZ4 when `encoding` is IX_PAYLOAD_SHUFFLE_LZ4 and the
 * block is smaller than the raw bytes; otherwise the raw bytes themselves (Raw).
 * `*used_encoding` is the payload's encoding, `*wire_len` its length; raw_len is
 * `raw_len`.  `wire_cap` >= ix_payload_max_encoded_len(raw_len) always suffices. */
int ix_payload_encode(uint32_t encoding, const uint8_t* raw, size_t raw_len, uint8_t* wire, size_t wire_cap,
                      size_t* wire_len, uint32_t* used_encoding);

/* PayloadDecoder::decode_and_add with its bounded-decode checks, in the reference's
 * order: size cap, raw_len, supported encoding, decompression into exactly raw_len bytes,
 * short output.  `acc` is width * height Vec3 sums (3 floats per pixel); a decoded pixel
 * is added only when every component is finite and >= 0, `*dropped` counts the others.
 * On an error nothing is added. */
int ix_payload_decode_and_add(uint32_t encoding, uint32_t raw_len, const uint8_t* wire, size_t wire_len,
                              uint32_t width, uint32_t height, float* acc, uint32_t* dropped);

/* PayloadDecoder::decode_to_vec: the decoded Vec3 values into `out` (3 floats per pixel). */
int ix_payload_decode(uint32_t encoding, uint32_t raw_len, const uint8_t* wire, size_t wire_len, uint32_t width,
                      uint32_t height, float* out);

/* Device forms for a lane whose sums live on the GPU.  Encode: `d_sums` (width * height *
 * 3 doubles, device) rounded to f32 and, for LZ4, byte-shuffled by one kernel, copied to
 * the host and compressed.  Decode: the block decompressed on the host into pinned
 * memory, copied to the device, and one kernel unshuffles, applies the valid-sample rule
 * and adds into `d_acc` (width * height * 3 floats, device).  Both run on `stream`
 * (NULL: the backend's own) and return when their results are complete. */
int ix_payload_encode_device(struct ix_backend* b, uint32_t encoding, const double* d_sums, uint32_t width,
                             uint32_t height, uint8_t* wire, size_t wire_cap, size_t* wire_len,
                             uint32_t* used_encoding, void* stream);
int ix_payload_decode_and_add_device(struct ix_backend* b, uint32_t encoding, uint32_t raw_len, const uint8_t* wire,
                                     size_t wire_len, uint32_t width, uint32_t height, float* d_acc,
                                     uint32_t* dropped, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IX_RADIANCE_H */
