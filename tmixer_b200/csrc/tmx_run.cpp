// tmx_run -- C++ host driver over the C ABI: the counterpart of the
// reference's main() (Tmixer.cpp:10413-10490).  It runs one case on one GPU,
// reports progress and the outlet mixing index every `--every` steps (the
// reference writes its files every time_step = 1000 steps, :10476), and writes
// the final fields as raw little-endian doubles plus the mixing rows as text.
//
//   tmx_run [--case reference | --case w --W 32 --umax 0.05 --tauf 0.56 --tauc 0.6 --k 1e-3 --rho 1]
//           [--steps N] [--every M] [--out DIR] [--files] [--domain-every D] [--device D]
//           [--precision fp64|fp32|fp16]
//
// With --files (and --out) it also writes the reference's Tecplot files into
// DIR at the reference's moments: after step itr+1 for itr % every == 0,
// Data_P_V_C<itr>.dat, Pressure_<itr>.dat and MixingQuality_<itr>.dat, plus
// Domain_Data_<itr>.dat when itr % domain-every == 0 (the reference's
// time_step 1000 and time_domaindata 5000, Tmixer.cpp:147-148, 10476-10486),
// and Data_P_V_C100.dat after step 101.
//
// Output (with --out): DIR/fields.bin = int32 {inx, iny, nz, mnx, mny, ia, ib,
// steps} then rho, ux, uy, uz, cA, cB, cC of the inlet box and of the mixing
// box, each in [i][j][k] order; DIR/mixing.txt = one row per line.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tmx.h"

static int die(const char* what)
{
    std::fprintf(stderr, "tmx_run: %s: %s\n", what, tmx_last_error());
    return 1;
}

int main(int argc, char** argv)
{
    std::string kind = "reference", out;
    int W = 32, device = 0;
    bool files = false;
    int precision = TMX_FP64;
    long long steps = -1, every = 1000, domain_every = 5000;
    double umax = 0.05, tauf = 0.56, tauc = 0.6, k = 1e-3, rho = 1.0;
    for (int a = 1; a < argc; a++) {
        auto next = [&](const char* name) -> const char* {
            if (a + 1 >= argc) {
                std::fprintf(stderr, "tmx_run: %s needs a value\n", name);
                std::exit(2);
            }
            return argv[++a];
        };
        if (!std::strcmp(argv[a], "--case")) kind = next("--case");
        else if (!std::strcmp(argv[a], "--W")) W = std::atoi(next("--W"));
        else if (!std::strcmp(argv[a], "--umax")) umax = std::atof(next("--umax"));
        else if (!std::strcmp(argv[a], "--tauf")) tauf = std::atof(next("--tauf"));
        else if (!std::strcmp(argv[a], "--tauc")) tauc = std::atof(next("--tauc"));
        else if (!std::strcmp(argv[a], "--k")) k = std::atof(next("--k"));
        else if (!std::strcmp(argv[a], "--rho")) rho = std::atof(next("--rho"));
        else if (!std::strcmp(argv[a], "--steps")) steps = std::atoll(next("--steps"));
        else if (!std::strcmp(argv[a], "--every")) every = std::atoll(next("--every"));
        else if (!std::strcmp(argv[a], "--out")) out = next("--out");
        else if (!std::strcmp(argv[a], "--files")) files = true;
        else if (!std::strcmp(argv[a], "--precision")) {
            const char* v = next("--precision");
            precision = !std::strcmp(v, "fp32") ? TMX_FP32 : !std::strcmp(v, "fp16") ? TMX_FP16 : TMX_FP64;
            if (std::strcmp(v, "fp64") && std::strcmp(v, "fp32") && std::strcmp(v, "fp16")) {
                std::fprintf(stderr, "tmx_run: --precision is fp64, fp32 or fp16\n");
                return 2;
            }
        }
        else if (!std::strcmp(argv[a], "--domain-every")) domain_every = std::atoll(next("--domain-every"));
        else if (!std::strcmp(argv[a], "--device")) device = std::atoi(next("--device"));
        else {
            std::fprintf(stderr, "usage: %s [--case reference|w] [--W n] [--steps n] [--every n] [--out dir]\n",
                         argv[0]);
            return 2;
        }
    }
    tmx_case c;
    if (kind == "reference") {
        if (tmx_case_reference(&c)) return die("case");
        if (steps < 0) steps = 100001;  // the reference loops itr = 0..time (Tmixer.cpp:10467)
    } else {
        if (tmx_case_wlayout(W, umax, tauf, tauc, k, rho, &c)) return die("case");
        if (steps < 0) steps = 1000;
    }
    if (every <= 0) every = steps;
    c.precision = precision;
    tmx_handle* h = nullptr;
    if (tmx_create(&c, device, &h)) return die("create");
    const auto t0 = std::chrono::steady_clock::now();
    if (tmx_init(h)) return die("init");
    const long long nodes = (long long)c.inx * c.iny * c.nz + (long long)c.mnx * c.mny * c.nz;
    std::printf("nx:%d ny:%d nz:%d ia:%d ib:%d nodes:%lld steps:%lld\n", c.inx, c.iny + c.mny, c.nz, c.ia,
                c.ia + c.mnx - 1, nodes, steps);
    std::vector<double> rows((size_t)(c.mny + c.iny) * 7);
    double im[3];
    if (files && out.empty()) {
        std::fprintf(stderr, "tmx_run: --files needs --out\n");
        return 2;
    }
    if (domain_every <= 0) domain_every = every;
    // the reference's files after step itr+1 (itr counts from 0)
    auto write_files = [&](long long itr) -> int {
        char name[64];
        const struct {
            int kind;
            const char* fmt;
            bool when;
        } outs[4] = {{TMX_FILE_PVC, "Data_P_V_C%lld.dat", itr % every == 0 || itr == 100},
                     {TMX_FILE_PRESSURE, "Pressure_%lld.dat", itr % every == 0},
                     {TMX_FILE_MIXING, "MixingQuality_%lld.dat", itr % every == 0},
                     {TMX_FILE_DOMAIN, "Domain_Data_%lld.dat", itr % every == 0 && itr % domain_every == 0}};
        for (const auto& o : outs) {
            if (!o.when) continue;
            std::snprintf(name, sizeof name, o.fmt, itr);
            if (tmx_write_file(h, o.kind, (out + "/" + name).c_str())) return die("write_file");
        }
        return 0;
    };
    long long done = 0;
    while (done < steps) {
        long long n = std::min(every, steps - done);
        if (files) {  // stop at the next step after which the reference writes
            const long long itr = done;  // the loop index of the next step
            long long stop = itr % every == 0 ? itr : (itr / every + 1) * every;
            if (itr <= 100 && stop > 100) stop = 100;
            n = std::min(stop - itr + 1, steps - done);
        }
        if (tmx_step(h, (int)n)) return die("step");
        done += n;
        if (files) {
            const long long itr = done - 1;
            if (itr % every == 0 || itr == 100)
                if (write_files(itr)) return 1;
        }
        if (tmx_mixing(h, rows.data(), im)) return die("mixing");
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("step %lld  outlet I_A %.9g I_B %.9g I_C %.9g  %.1f MLUPS\n", done, im[0], im[1], im[2],
                    nodes * (double)done / s / 1e6);
        std::fflush(stdout);
    }
    if (!out.empty()) {
        std::string fp = out + "/fields.bin";
        FILE* f = std::fopen(fp.c_str(), "wb");
        if (!f) {
            std::perror(fp.c_str());
            return 1;
        }
        int hdr[8] = {c.inx, c.iny, c.nz, c.mnx, c.mny, c.ia, c.ia + c.mnx - 1, (int)steps};
        std::fwrite(hdr, sizeof(int), 8, f);
        for (int box = 0; box < 2; box++) {
            const size_t n = box == 0 ? (size_t)c.inx * c.iny * c.nz : (size_t)c.mnx * c.mny * c.nz;
            std::vector<double> buf(n);
            for (int fld = 0; fld < 7; fld++) {
                if (tmx_fields(h, box, fld, buf.data())) return die("fields");
                std::fwrite(buf.data(), sizeof(double), n, f);
            }
        }
        std::fclose(f);
        std::string mp = out + "/mixing.txt";
        FILE* m = std::fopen(mp.c_str(), "w");
        if (!m) {
            std::perror(mp.c_str());
            return 1;
        }
        for (int r = 0; r < c.mny + c.iny; r++) {
            const double* o = &rows[(size_t)r * 7];
            std::fprintf(m, "%d\t%.17g\t%.17g\t%.17g\t%.17g\t%.17g\t%.17g\n", (int)o[0], o[1], o[2], o[3], o[4], o[5],
                         o[6]);
        }
        std::fclose(m);
    }
    tmx_destroy(h);
    return 0;
}
