// leopard.cu -- Leopard GF(2^16) / GF(2^8) codecs (placeholder until the FFT kernels land).
#include "rsgpu_internal.h"

namespace rsgpu {
int leo_create(rsgpu_encoder *enc) {
    if (enc->k <= 0 || enc->p <= 0) return RS_ERR_INV_SHARD_NUM;
    if (enc->k + enc->p > 65536) return RS_ERR_MAX_SHARD_NUM;
    return RS_OK;
}
int leo_encode(rsgpu_encoder *, uint8_t *const *, size_t) { return RS_ERR_NOT_SUPPORTED; }
int leo_verify(rsgpu_encoder *, uint8_t *const *, size_t, int *) { return RS_ERR_NOT_SUPPORTED; }
int leo_reconstruct(rsgpu_encoder *, uint8_t **, const uint8_t *, size_t, int, uint8_t *) {
    return RS_ERR_NOT_SUPPORTED;
}
}  // namespace rsgpu
namespace rsgpu {
int leo_encode_enqueue(rsgpu_encoder *, uint8_t *const *, size_t) { return RS_ERR_NOT_SUPPORTED; }
int leo_reconstruct_enqueue(rsgpu_encoder *, uint8_t *const *, const uint8_t *, size_t, int) {
    return RS_ERR_NOT_SUPPORTED;
}
}  // namespace rsgpu
