// Field files in the reference's .D format and asynchronous dumps.
//
// Replaces the writers WRT_INSTANT_VARS_TG / WRT_INSTANT_VARS_FLOW_IO /
// WRT_INSTANT_VARS_THERMAL_IO (src/processing/WRT_VARS_TG.f90:13-100,
// src/processing/WRT_VARS_IO.f90:24-227) and the readers of
// ReStart_INSTANT_VARS_* (src/processing/RESTART_tg.f90:11-56,
// READ_INTP_3D_VARS.f90:20-80).  A .D file is a 40-byte header, int32[4]
// {NCL1, NCL2, NCL3, ITERG} then float64[3] {PhyTIME, REN, DT}, followed by
// the interior field float64 (NCL1, NCL2, NCL3) in Fortran order (no ghost
// planes); the name is <path>DNS_perixz_INSTANT_T<PhyTIME as ES15.9>_<X>.D
// with X = U, V, W, P and, with the thermal solver, T, D, H, M, K
// (TEMPERATURE, DENSITY, ENTHALPY, Viscousity, THERMCONDT).
//
// A dump is taken in two calls.  chapsim_dump_begin packs the interiors of
// the fields, and the device dt, into a snapshot buffer in HBM (2D copies
// on the context's stream, so in order with the steps; FP32 fields of the
// mixed-precision step are widened first), then copies the snapshot to
// pinned host memory on a stream of its own: the copy overlaps the steps
// the caller launches next.  chapsim_dump_write waits for that copy and
// writes the files.  A new dump waits (on the device) for the previous
// copy before it overwrites the snapshot.
#pragma once
#include <cstdio>
#include <string>

namespace {

constexpr int DUMP_FLOW = 4, DUMP_THERMAL = 5;
const char* const dump_suffix[DUMP_FLOW + DUMP_THERMAL] = {"_U.D", "_V.D", "_W.D", "_P.D", "_T.D",
                                                           "_D.D", "_H.D", "_M.D", "_K.D"};

int dump_nfields(const chapsim_ctx* ctx) { return DUMP_FLOW + (ctx->thermal ? DUMP_THERMAL : 0); }

// the padded (L, 0:M+1, N) device arrays of the dumped fields, in file order
void dump_sources(const chapsim_ctx* ctx, const double* src[DUMP_FLOW + DUMP_THERMAL]) {
    const Geo& g = ctx->g;
    src[0] = ctx->Q;
    src[1] = ctx->Q + g.FS;
    src[2] = ctx->Q + 2 * g.FS;
    src[3] = ctx->PR;
    if (ctx->thermal) {
        src[4] = ctx->tf.TEMP;
        src[5] = ctx->DEN;
        src[6] = ctx->tf.ENTH;
        src[7] = ctx->io.MU;
        src[8] = ctx->tf.KAP;
    }
}

// PhyTIME as Fortran's ES15.9 edit descriptor prints it for |exponent| < 100
std::string es15_9(double t) {
    char b[64];
    std::snprintf(b, sizeof b, "%.9E", t);
    return b;
}

}  // namespace

extern "C" {

int chapsim_write_dfile(const char* path, int32_t L, int32_t M, int32_t N, int32_t iterg, double time, double ren,
                        double dt, const double* field) {
    if (!path || !field || L <= 0 || M <= 0 || N <= 0)
        return fail(nullptr, CHAPSIM_ERR_BADARG, "chapsim_write_dfile: bad arguments");
    FILE* fh = std::fopen(path, "wb");
    if (!fh) return fail(nullptr, CHAPSIM_ERR_BADARG, std::string("cannot open ") + path + " for writing");
    const int32_t hi[4] = {L, M, N, iterg};
    const double hr[3] = {time, ren, dt};
    const size_t n = (size_t)L * M * N;
    bool ok = std::fwrite(hi, sizeof(int32_t), 4, fh) == 4 && std::fwrite(hr, sizeof(double), 3, fh) == 3 &&
              std::fwrite(field, sizeof(double), n, fh) == n;
    ok = (std::fclose(fh) == 0) && ok;
    if (!ok) return fail(nullptr, CHAPSIM_ERR_BADARG, std::string("short write to ") + path);
    return CHAPSIM_OK;
}

int chapsim_read_dfile(const char* path, int32_t* dims4, double* reals3, double* field, int64_t capacity) {
    if (!path || !dims4 || !reals3) return fail(nullptr, CHAPSIM_ERR_BADARG, "chapsim_read_dfile: bad arguments");
    FILE* fh = std::fopen(path, "rb");
    if (!fh) return fail(nullptr, CHAPSIM_ERR_BADARG, std::string("cannot open ") + path);
    int32_t hi[4];
    double hr[3];
    if (std::fread(hi, sizeof(int32_t), 4, fh) != 4 || std::fread(hr, sizeof(double), 3, fh) != 3) {
        std::fclose(fh);
        return fail(nullptr, CHAPSIM_ERR_BADARG, std::string(path) + ": truncated header");
    }
    std::fseek(fh, 0, SEEK_END);
    const long long bytes = std::ftell(fh);
    const long long n = (long long)hi[0] * hi[1] * hi[2];
    if (hi[0] <= 0 || hi[1] <= 0 || hi[2] <= 0 || bytes != 40 + 8 * n) {
        std::fclose(fh);
        return fail(nullptr, CHAPSIM_ERR_BADARG, std::string(path) + ": header dimensions do not match the payload");
    }
    for (int a = 0; a < 4; ++a) dims4[a] = hi[a];
    for (int a = 0; a < 3; ++a) reals3[a] = hr[a];
    if (field) {
        if (capacity < n) {
            std::fclose(fh);
            return fail(nullptr, CHAPSIM_ERR_BADARG, std::string(path) + ": the field does not fit the buffer");
        }
        std::fseek(fh, 40, SEEK_SET);
        const bool ok = std::fread(field, sizeof(double), (size_t)n, fh) == (size_t)n;
        std::fclose(fh);
        if (!ok) return fail(nullptr, CHAPSIM_ERR_BADARG, std::string(path) + ": short read");
        return CHAPSIM_OK;
    }
    std::fclose(fh);
    return CHAPSIM_OK;
}

int chapsim_dump_begin(chapsim_ctx_t* ctx) {
    if (!ctx) return fail(nullptr, CHAPSIM_ERR_BADARG, "null context");
    CK(cudaSetDevice(ctx->device));
    const Geo& g = ctx->g;
    const int nf = dump_nfields(ctx);
    const size_t n = (size_t)g.L * g.M * g.N;
    const size_t words = (size_t)nf * n + 1;  // the fields, then dt
    if (ctx->dump_words != words) {
        if (ctx->dump_pending) CK(cudaEventSynchronize(ctx->dump_done));
        ctx->dump_pending = false;
        cudaFree(ctx->dump_dev);
        if (ctx->dump_host) cudaFreeHost(ctx->dump_host);
        ctx->dump_dev = nullptr;
        ctx->dump_host = nullptr;
        ctx->dump_words = 0;
        CK(cudaMalloc(&ctx->dump_dev, words * sizeof(double)));
        CK(cudaMallocHost(&ctx->dump_host, words * sizeof(double)));
        ctx->dump_words = words;
        if (!ctx->dump_stream) CK(cudaStreamCreateWithFlags(&ctx->dump_stream, cudaStreamNonBlocking));
        if (!ctx->dump_snap) CK(cudaEventCreateWithFlags(&ctx->dump_snap, cudaEventDisableTiming));
        if (!ctx->dump_done) CK(cudaEventCreateWithFlags(&ctx->dump_done, cudaEventDisableTiming));
    }
    cudaStream_t s = ctx->stream;
    if (ctx->dump_pending) CK(cudaStreamWaitEvent(s, ctx->dump_done, 0));  // the previous copy has left the snapshot
    if (ctx->prec == CHAPSIM_PREC_MIXED) {
        int rc = mixed_to_staging(ctx, true, true, false);
        if (rc) return rc;
    }
    const double* src[DUMP_FLOW + DUMP_THERMAL] = {};
    dump_sources(ctx, src);
    const size_t row = (size_t)g.L * sizeof(double);
    for (int f = 0; f < nf; ++f)  // rows j = 1..M of every plane k: one 2D copy
        CK(cudaMemcpy2DAsync(ctx->dump_dev + f * n, (size_t)g.M * row, src[f] + g.L, (size_t)(g.M + 2) * row,
                             (size_t)g.M * row, (size_t)g.N, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(ctx->dump_dev + nf * n, &ctx->st->dt, sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaEventRecord(ctx->dump_snap, s));
    CK(cudaStreamWaitEvent(ctx->dump_stream, ctx->dump_snap, 0));
    CK(cudaMemcpyAsync(ctx->dump_host, ctx->dump_dev, words * sizeof(double), cudaMemcpyDeviceToHost, ctx->dump_stream));
    CK(cudaEventRecord(ctx->dump_done, ctx->dump_stream));
    ctx->dump_pending = true;
    ctx->dump_nf = nf;
    return CHAPSIM_OK;
}

int chapsim_dump_write(chapsim_ctx_t* ctx, const char* path_prefix, int32_t iterg, double time, double ren,
                       double* dt_out) {
    if (!ctx || !path_prefix) return fail(ctx, CHAPSIM_ERR_BADARG, "chapsim_dump_write: bad arguments");
    if (!ctx->dump_pending) return fail(ctx, CHAPSIM_ERR_BADARG, "no dump in flight: call chapsim_dump_begin first");
    CK(cudaSetDevice(ctx->device));
    CK(cudaEventSynchronize(ctx->dump_done));
    ctx->dump_pending = false;
    const Geo& g = ctx->g;
    const size_t n = (size_t)g.L * g.M * g.N;
    const double dt = ctx->dump_host[(size_t)ctx->dump_nf * n];
    if (dt_out) *dt_out = dt;
    const std::string stem = std::string(path_prefix) + es15_9(time);
    for (int f = 0; f < ctx->dump_nf; ++f) {
        const std::string path = stem + dump_suffix[f];
        int rc = chapsim_write_dfile(path.c_str(), g.L, g.M, g.N, iterg, time, ren, dt, ctx->dump_host + f * n);
        if (rc) return fail(ctx, rc, g_init_error);
    }
    return CHAPSIM_OK;
}

}  // extern "C"
