// transcript_capi.cpp -- C ABI over the host Poseidon2 transcript and the CCS
// matrix digest (no GPU needed).
#include <new>
#include "../../include/neo_gpu.h"
#include "abi_guard.h"
#include "transcript.h"

struct neo_transcript {
    neo::Transcript tr;
    explicit neo_transcript(const char* l) : tr(l) {}
};

static int neo_transcript_new_impl_abi(const char* app_label, neo_transcript** out) {
    if (!app_label || !out) return NEO_ERR_ARG;
    *out = new (std::nothrow) neo_transcript(app_label);
    return *out ? NEO_OK : NEO_ERR_OOM;
}
extern "C" int neo_transcript_new(const char* app_label, neo_transcript** out) { NEO_ABI_GUARD(neo_transcript_new_impl_abi(app_label, out)) }
static int neo_transcript_destroy_impl_abi(neo_transcript* t) {
    if (!t) return NEO_ERR_ARG;
    delete t;
    return NEO_OK;
}
extern "C" int neo_transcript_destroy(neo_transcript* t) { NEO_ABI_GUARD(neo_transcript_destroy_impl_abi(t)) }
static int neo_transcript_append_message_impl_abi(neo_transcript* t, const char* label, const uint8_t* msg, size_t len) {
    if (!t || !label || (len && !msg)) return NEO_ERR_ARG;
    t->tr.append_message(label, msg, len);
    return NEO_OK;
}
extern "C" int neo_transcript_append_message(neo_transcript* t, const char* label, const uint8_t* msg, size_t len) { NEO_ABI_GUARD(neo_transcript_append_message_impl_abi(t, label, msg, len)) }
static int neo_transcript_append_fields_impl_abi(neo_transcript* t, const char* label, const uint64_t* fs, size_t n) {
    if (!t || !label || (n && !fs)) return NEO_ERR_ARG;
    t->tr.append_fields(label, fs, n);
    return NEO_OK;
}
extern "C" int neo_transcript_append_fields(neo_transcript* t, const char* label, const uint64_t* fs, size_t n) { NEO_ABI_GUARD(neo_transcript_append_fields_impl_abi(t, label, fs, n)) }
static int neo_transcript_append_u64s_impl_abi(neo_transcript* t, const char* label, const uint64_t* us, size_t n) {
    if (!t || !label || (n && !us)) return NEO_ERR_ARG;
    t->tr.append_u64s(label, us, n);
    return NEO_OK;
}
extern "C" int neo_transcript_append_u64s(neo_transcript* t, const char* label, const uint64_t* us, size_t n) { NEO_ABI_GUARD(neo_transcript_append_u64s_impl_abi(t, label, us, n)) }
static int neo_transcript_challenge_field_impl_abi(neo_transcript* t, const char* label, uint64_t* out) {
    if (!t || !label || !out) return NEO_ERR_ARG;
    *out = t->tr.challenge_field(label);
    return NEO_OK;
}
extern "C" int neo_transcript_challenge_field(neo_transcript* t, const char* label, uint64_t* out) { NEO_ABI_GUARD(neo_transcript_challenge_field_impl_abi(t, label, out)) }
static int neo_transcript_challenge_fields_impl_abi(neo_transcript* t, const char* label, size_t n, uint64_t* out) {
    if (!t || !label || (n && !out)) return NEO_ERR_ARG;
    t->tr.challenge_fields(label, n, out);
    return NEO_OK;
}
extern "C" int neo_transcript_challenge_fields(neo_transcript* t, const char* label, size_t n, uint64_t* out) { NEO_ABI_GUARD(neo_transcript_challenge_fields_impl_abi(t, label, n, out)) }
static int neo_transcript_digest32_impl_abi(neo_transcript* t, uint8_t* out) {
    if (!t || !out) return NEO_ERR_ARG;
    t->tr.digest32(out);
    return NEO_OK;
}
extern "C" int neo_transcript_digest32(neo_transcript* t, uint8_t* out) { NEO_ABI_GUARD(neo_transcript_digest32_impl_abi(t, out)) }
static int neo_transcript_state_impl_abi(const neo_transcript* t, uint64_t* st8) {
    if (!t || !st8) return NEO_ERR_ARG;
    for (int i = 0; i < 8; i++) st8[i] = t->tr.state()[i];
    return NEO_OK;
}
extern "C" int neo_transcript_state(const neo_transcript* t, uint64_t* st8) { NEO_ABI_GUARD(neo_transcript_state_impl_abi(t, st8)) }
