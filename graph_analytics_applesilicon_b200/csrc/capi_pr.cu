// capi_pr.cu -- extern "C" entry points of PageRank (include/graph_b200.h).
#include <cstring>
#include <memory>

#include "capi_util.hpp"
#include "graph_prep.cuh"
#include "pagerank.hpp"

using namespace gb;

extern "C" {

void gb_pr_default_options(gb_pr_options* o) {
    if (!o) return;
    *o = gb_pr_options{};
    o->damping = 0.85f;  // src/metal/pagerank_gpu.hpp:27-36 defaults
    o->iters = 20;
    o->tol = 0;
    o->tol_rel = 0;
    o->tg = 256;
    o->small_max = 16;
    o->large_min = 256;
    o->inplace = 0;
}

int gb_pr_create(uint64_t n, const uint32_t* out_row_ptr, const uint32_t* out_col_idx, uint64_t out_m,
                 const uint32_t* in_row_ptr, const uint32_t* in_col_idx, uint64_t in_m, const uint32_t* outdeg,
                 gb_pr** out) {
    return guard([&] {
        GB_REQUIRE(out, "null handle output");
        GB_REQUIRE(n < 0xFFFFFFFFull, "too many vertices for uint32 ids");
        GB_REQUIRE(outdeg || n == 0, "null out-degrees");
        GB_REQUIRE(out_row_ptr || in_row_ptr, "need the out-CSR, the in-CSR or both");
        auto h = std::make_unique<gb_pr>();
        h->n = n;
        if (out_row_ptr) {
            GB_REQUIRE(out_m == 0 || out_col_idx, "null out col_idx");
            GB_REQUIRE(out_row_ptr[0] == 0 && out_row_ptr[n] == out_m, "out row_ptr inconsistent with m");
            h->hasOut = true;
            h->mOut = out_m;
            h->rowOut.ensure(n + 1);
            h->colOut.ensure(out_m + 4);
            GB_CUDA(cudaMemcpy(h->rowOut.get(), out_row_ptr, (n + 1) * 4, cudaMemcpyHostToDevice));
            if (out_m) GB_CUDA(cudaMemcpy(h->colOut.get(), out_col_idx, out_m * 4, cudaMemcpyHostToDevice));
            checkDeviceCsr(h->rowOut.get(), h->colOut.get(), n, out_m, 0);
        }
        if (in_row_ptr) {
            GB_REQUIRE(in_m == 0 || in_col_idx, "null in col_idx");
            GB_REQUIRE(in_row_ptr[0] == 0 && in_row_ptr[n] == in_m, "in row_ptr inconsistent with m");
            h->hasIn = true;
            h->mIn = in_m;
            h->rowIn.ensure(n + 1);
            h->colIn.ensure(in_m + 4);
            GB_CUDA(cudaMemset(h->colIn.get(), 0, (in_m + 4) * 4));
            GB_CUDA(cudaMemcpy(h->rowIn.get(), in_row_ptr, (n + 1) * 4, cudaMemcpyHostToDevice));
            if (in_m) GB_CUDA(cudaMemcpy(h->colIn.get(), in_col_idx, in_m * 4, cudaMemcpyHostToDevice));
            checkDeviceCsr(h->rowIn.get(), h->colIn.get(), n, in_m, 0);
            h->hostRowIn.assign(in_row_ptr, in_row_ptr + n + 1);
            h->hostColIn.assign(in_col_idx, in_col_idx + in_m);
        }
        h->outdeg.ensure(n + 1);
        if (n) GB_CUDA(cudaMemcpy(h->outdeg.get(), outdeg, n * 4, cudaMemcpyHostToDevice));
        h->hostOutdeg.assign(outdeg, outdeg + n);
        for (int i = 0; i < 2; ++i) {
            h->r[i].ensure(n + 1);
            h->contrib[i].ensure(n + 4);  // the blocked pull copies whole 16-byte groups past n
        }
        h->ctl.ensure(1);
        h->partF.ensure(2 * 4096);
        h->partD.ensure(3 * 4096);
        *out = h.release();
    });
}

int gb_pr_destroy(gb_pr* h) {
    return guard([&] {
        if (h) {
            cudaStreamSynchronize(h->stream.s);
            delete h;
        }
    });
}

int gb_pr_prepare_adaptive(gb_pr* h, uint32_t small_max, uint32_t large_min) {
    return guard([&] {
        GB_REQUIRE(h, "null handle");
        h->prepareAdaptive(small_max, large_min);
    });
}

int gb_pr_prepare_gs(gb_pr* h, uint32_t pair_max_outdeg) {
    return guard([&] {
        GB_REQUIRE(h, "null handle");
        h->prepareGS(pair_max_outdeg);
    });
}

int gb_pr_gs_info(const gb_pr* h, int* colored, uint64_t* sets, uint64_t* deferred) {
    return guard([&] {
        GB_REQUIRE(h, "null handle");
        if (colored) *colored = h->gsColored ? 1 : 0;
        if (sets) *sets = h->gsSetStart.empty() ? 0 : h->gsSetStart.size() - 1;
        if (deferred) *deferred = h->gsDeferred;
    });
}

int gb_pr_run(gb_pr* h, int variant, const gb_pr_options* opt, gb_pr_result* res) {
    return guard([&] {
        GB_REQUIRE(h, "null handle");
        gb_pr_options o;
        gb_pr_default_options(&o);
        if (opt) o = *opt;
        gb_pr_result r = h->run(variant, o);
        if (res) *res = r;
    });
}

int gb_pr_ranks(gb_pr* h, float* out_host) {
    return guard([&] {
        GB_REQUIRE(h && (out_host || h->n == 0), "null argument");
        if (h->n) h->ranks(out_host);
    });
}

int gb_pr_ranks_f64(gb_pr* h, double* out_host) {
    return guard([&] {
        GB_REQUIRE(h && (out_host || h->n == 0), "null argument");
        if (h->n) h->ranks64(out_host);
    });
}

void* gb_pr_stream(const gb_pr* h) { return h ? (void*)h->stream.s : nullptr; }

}  // extern "C"
