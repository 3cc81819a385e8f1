// mp_serve.cu -- request serving with continuous batching (see include/mathpub_gpu.h).
#include "mp_common.cuh"

extern "C" {
int mp_serve_open(mp_handle *h, const mp_serve_opts *, mp_server **out)
{
    if (out) *out = nullptr;
    return mp_set_error(h, MP_EINVAL, "serving not built yet");
}
int mp_serve_submit_range(mp_server *, uint64_t, uint64_t, uint64_t *) { return MP_EINVAL; }
int mp_serve_submit_bpsw(mp_server *, const uint64_t *, uint32_t, uint8_t *, uint64_t *) { return MP_EINVAL; }
int mp_serve_poll(mp_server *, uint64_t, mp_serve_result *, int) { return MP_EINVAL; }
int mp_serve_close(mp_server *) { return MP_EINVAL; }
}
