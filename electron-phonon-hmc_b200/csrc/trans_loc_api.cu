// Drop-in surface of the static-disorder mode: hist_trans_loc and
// run_trans_loc with the reference's prototypes (simulation/organic_trans_loc.h:4-6)
// over the ephmc_tl handles of trans_loc.cu.
//
// The bond fields come from the host program's MT19937-64 stream (its
// random_vector, or the library's copy of it), drawn in the reference's order:
// one random_vector of 3V normals at the start of every sample.  run_trans_loc
// draws the fields of all samples first and hands them to the GPU in batches,
// so several samples are diagonalised at once; the files it writes have the
// reference's formats (fprint_results per sample, fwrite_sigma at the end).
#include "ephmc_internal.cuh"
#include "../../include/ephmc_organic.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

using namespace ephmc;

namespace {

std::mutex g_tl_mu;
std::map<std::tuple<int, unsigned, unsigned, uint64_t>, ephmc_tl *> g_tl_reg;

uint64_t tl_hash_nnt(const unsigned *nnt, unsigned ns) {
    uint64_t h = 1469598103934665603ULL;
    for (size_t i = 0; i < 6 * (size_t)ns; ++i) {
        h ^= nnt[i];
        h *= 1099511628211ULL;
    }
    return h;
}

// samples diagonalised concurrently by the drop-in: EPHMC_TL_LANES, default 2
// (two lanes measured 8% faster than one on a 64x64 lattice, four no faster than two)
unsigned tl_lanes() {
    if (const char *s = std::getenv("EPHMC_TL_LANES")) {
        const long v = std::strtol(s, nullptr, 10);
        if (v >= 1 && v <= 16) return (unsigned)v;
    }
    return 2;
}

ephmc_tl *tl_for(const unsigned *nnt, unsigned ns, unsigned nbins, const double *t, const double *kappa, double mu,
                 const double *contr_mat) {
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, ns, nbins, tl_hash_nnt(nnt, ns));
    std::lock_guard<std::mutex> l(g_tl_mu);
    auto it = g_tl_reg.find(key);
    if (it != g_tl_reg.end()) {
        tl_set_params(it->second, t, kappa, mu, contr_mat);
        return it->second;
    }
    ephmc_tl *tl = nullptr;
    if (tl_create_nnt(&tl, nnt, ns, nbins, t, kappa, mu, contr_mat, tl_lanes(), dev) != EPHMC_OK) return nullptr;
    g_tl_reg[key] = tl;
    return tl;
}

void tl_report(const char *fn) { std::fprintf(stderr, "ephmc %s: %s\n", fn, ephmc_last_error_message()); }

bool tl_devp(const void *p) {
    cudaPointerAttributes a{};
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// fprint_results(out, res, 1, 1) (simulation/organic_aux.c:62-70)
void print_result(FILE *out, double v) {
    if (!out) return;
    std::fprintf(out, "%.15g\t", v);
    std::fprintf(out, "\n");
    std::fflush(out);
}

// fwrite_sigma (simulation/organic_aux.c:82-90): unsigned n, double width, double[n]
void write_sigma(const char *name, const double *greens, double width, unsigned n) {
    if (!name) return;
    FILE *out = std::fopen(name, "w");
    if (!out) {
        std::fprintf(stderr, "ephmc run_trans_loc: cannot open %s\n", name);
        return;
    }
    std::fwrite(&n, sizeof(unsigned), 1, out);
    std::fwrite(&width, sizeof(double), 1, out);
    std::fwrite(greens, sizeof(double), n, out);
    std::fclose(out);
}

}  // namespace

extern "C" {

// hist_trans_loc (simulation/organic_trans_loc.c:25-83): one sample.  x is the
// caller's work array; x[0 .. 3ns) receives the bond field as in the reference.
void hist_trans_loc(double *x, double *t, double *kappa, double mu, double *contr_mat, unsigned *nnt, unsigned ns,
                    unsigned nn, unsigned nt, double width, double *results, double *greens, FILE *res_out) {
    if (nn != 6) {
        set_status(EPHMC_ERR_LATTICE, "hist_trans_loc: only the triangular lattice (nn = 6) is supported");
        return tl_report("hist_trans_loc");
    }
    const unsigned dim = ns * 3;
    std::vector<double> xh(dim);
    dropin_rng_normals(xh.data(), dim);
    if (tl_devp(x))
        cudaMemcpy(x, xh.data(), sizeof(double) * dim, cudaMemcpyHostToDevice);
    else
        std::copy(xh.begin(), xh.end(), x);
    std::vector<unsigned> nh(6 * (size_t)ns);
    if (tl_devp(nnt))
        cudaMemcpy(nh.data(), nnt, sizeof(unsigned) * 6 * ns, cudaMemcpyDeviceToHost);
    else
        std::copy(nnt, nnt + 6 * (size_t)ns, nh.begin());
    ephmc_tl *tl = tl_for(nh.data(), ns, nt, t, kappa, mu, contr_mat);
    if (!tl) return tl_report("hist_trans_loc");
    double z = 0;
    if (ephmc_tl_run(tl, xh.data(), 1, width, greens, &z) != EPHMC_OK) return tl_report("hist_trans_loc");
    if (tl_devp(results))
        cudaMemcpy(results, &z, sizeof(double), cudaMemcpyHostToDevice);
    else
        results[0] = z;
    print_result(res_out, z);
}

unsigned ephmc_run_trans_loc_seeded(unsigned long long seed, double *greens, unsigned l1, unsigned l2, unsigned nt,
                                    double *t, double *kappa, double mu, double *contr_mat, unsigned meas,
                                    const char *res_name, const char *corr_name) {
    const unsigned ns = l1 * l2, dim = 3 * ns;
    std::vector<unsigned> nnt(12 * (size_t)ns);
    triangular_lattice(l1, l2, nnt.data());
    double *results = greens + nt;
    ephmc_tl *tl = tl_for(nnt.data(), ns, nt, t, kappa, mu, contr_mat);
    if (!tl) {
        tl_report("run_trans_loc");
        return 0;
    }
    FILE *res_out = res_name ? std::fopen(res_name, "a") : nullptr;
    dropin_rng_seed(seed);
    // run_trans_loc's width, summed in its order (simulation/organic_trans_loc.c:99-100)
    double width = -2 * mu / nt;
    for (unsigned i = 0; i < 3; i++) width += 8 * std::fabs(kappa[i]) / nt;
    // fields of up to 64 samples per batch, drawn in sample order
    const unsigned batch = std::max(1u, std::min(meas, 64u));
    std::vector<double> xs((size_t)batch * dim);
    for (unsigned s0 = 0; s0 < meas; s0 += batch) {
        const unsigned nb = std::min(batch, meas - s0);
        for (unsigned s = 0; s < nb; ++s) dropin_rng_normals(xs.data() + (size_t)s * dim, dim);
        if (ephmc_tl_run(tl, xs.data(), nb, width, greens, results + s0) != EPHMC_OK) {
            tl_report("run_trans_loc");
            if (res_out) std::fclose(res_out);
            return 0;
        }
        for (unsigned s = 0; s < nb; ++s) print_result(res_out, results[s0 + s]);
    }
    for (unsigned k = 0; k < nt; k++) greens[k] /= meas;
    write_sigma(corr_name, greens, width, nt);
    if (res_out) std::fclose(res_out);
    return meas + nt;
}

// run_trans_loc (simulation/organic_trans_loc.c:85-114), seeded with time(NULL)
// as the reference, or with the value of the environment variable EPHMC_SEED
unsigned run_trans_loc(double *greens, unsigned l1, unsigned l2, unsigned nt, double *t, double *kappa, double mu,
                       double *contr_mat, unsigned meas, const char *res_name, const char *corr_name) {
    unsigned long long seed = (unsigned long long)std::time(nullptr);
    if (const char *s = std::getenv("EPHMC_SEED")) seed = std::strtoull(s, nullptr, 10);
    return ephmc_run_trans_loc_seeded(seed, greens, l1, l2, nt, t, kappa, mu, contr_mat, meas, res_name, corr_name);
}

}  // extern "C"
