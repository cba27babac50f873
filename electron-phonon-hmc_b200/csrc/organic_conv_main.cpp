// organic_conv on the GPU library: the command line, input parsing and output
// format of the reference's program (simulation/organic_conv.c:123-164), with
// the smearing and the Euclidean-time transform computed by
// ephmc_conv_sigma_w / ephmc_conv_sigma_t.
//
//   organic_conv greens.bin smear.txt greens_smeared.csv [corr_smeared.csv]
//
// greens.bin: unsigned n, double h, double sigma[n] (fwrite_sigma layout,
// simulation/organic_aux.c:82-90).  smear.txt: beta, nt, then the smearing
// widths in physical units (fscan_array, organic_aux.c:121-141).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/ephmc.h"

namespace {

bool read_greens(const char *name, double *h, std::vector<double> &sigma) {
    FILE *in = std::fopen(name, "rb");
    if (!in) return false;
    unsigned n = 0;
    bool ok = std::fread(&n, sizeof(unsigned), 1, in) == 1 && std::fread(h, sizeof(double), 1, in) == 1;
    if (ok) {
        sigma.resize(n);
        ok = std::fread(sigma.data(), sizeof(double), n, in) == n;
    }
    std::fclose(in);
    return ok;
}

bool read_smear(const char *name, double *beta, unsigned *nt, std::vector<double> &w) {
    FILE *in = std::fopen(name, "r");
    if (!in) return false;
    bool ok = std::fscanf(in, "%lg ", beta) == 1 && std::fscanf(in, "%u ", nt) == 1;
    double v;
    while (ok && std::fscanf(in, "%lg ", &v) > 0) w.push_back(v);
    std::fclose(in);
    return ok;
}

int fail(const char *what) {
    std::fprintf(stderr, "organic_conv: %s: %s\n", what, ephmc_last_error_message());
    return 1;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 4 && argc != 5) {
        std::printf("Error! 3 or 4 files needed: greens data, list of smearing widths, frequency output, opt. time "
                    "output.\n");
        return 0;
    }
    double h = 0, beta = 0;
    unsigned nt = 0;
    std::vector<double> sigma, widths;
    if (!read_greens(argv[1], &h, sigma)) {
        std::fprintf(stderr, "organic_conv: cannot read %s\n", argv[1]);
        return 1;
    }
    if (!read_smear(argv[2], &beta, &nt, widths)) {
        std::fprintf(stderr, "organic_conv: cannot read %s\n", argv[2]);
        return 1;
    }
    const unsigned n = (unsigned)sigma.size(), ns = (unsigned)widths.size();
    for (double &w : widths) w *= beta;
    FILE *out_w = std::fopen(argv[3], "w");
    if (!out_w) {
        std::fprintf(stderr, "organic_conv: cannot open %s\n", argv[3]);
        return 1;
    }
    if (ns > 0) {
        std::vector<double> sw((size_t)n * ns);
        if (ephmc_conv_sigma_w(sigma.data(), n, h, widths.data(), ns, sw.data()) != EPHMC_OK)
            return fail("ephmc_conv_sigma_w");
        for (unsigned i = 0; i < n; i++) {
            std::fprintf(out_w, "%g\t", i * h / beta);
            for (unsigned k = 0; k < ns; k++) std::fprintf(out_w, "%g\t", sw[(size_t)i * ns + k]);
            std::fprintf(out_w, "\n");
        }
    } else {
        for (unsigned i = 0; i < n; i++) std::fprintf(out_w, "%g\t\n", i * h / beta);
    }
    std::fclose(out_w);
    if (argc > 4) {
        FILE *out_t = std::fopen(argv[4], "w");
        if (!out_t) {
            std::fprintf(stderr, "organic_conv: cannot open %s\n", argv[4]);
            return 1;
        }
        std::vector<double> st(((size_t)nt / 2 + 1) * (ns ? ns : 1));
        if (ns > 0 && nt > 0 && ephmc_conv_sigma_t(sigma.data(), n, h, widths.data(), ns, nt, 0, st.data()) != EPHMC_OK)
            return fail("ephmc_conv_sigma_t");
        for (unsigned i = 0; i <= nt / 2; i++) {
            std::fprintf(out_t, "%g\t", (double)i / nt);
            for (unsigned k = 0; k < ns; k++) std::fprintf(out_t, "%g\t", st[(size_t)i * ns + k]);
            std::fprintf(out_t, "\n");
        }
        std::fclose(out_t);
    }
    return 0;
}
