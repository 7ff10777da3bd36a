// gsb2: the reference executor's command line (gsamp2.cpp:1-6, 126-227) on top of libgsb (include/gsb.h), so
// process-based callers (doped_sampler.py --bin, the cloud gate scripts, tests) can switch executors by path.
//
//   gsb2 plan sample N seed | sample2 N seed | prob strings | chain strings | hybrid strings seed
//   gsb2 plan prefix strings K outprefix | resume strings K seed dumpprefix... [--twist file]
//
// Output lines, their printf formats and the exit codes are the reference's.  The arena precision is complex64
// (the reference's default build) unless GSB_PRECISION=128 is set or the program is invoked under a name ending
// in "_c128" (the reference's -DGS_DOUBLE build); GSB_DEVICE picks the GPU.  Lines are evaluated in batches of
// GSB_BATCH (default 64) and printed and flushed after every batch.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gsb.h"

static int die(int rc) {
    if (rc == GSB_E_CUDA) {
        fprintf(stderr, "gsb2: %s\n", gsb_last_error());
        return 99;   // the reference GPU port's exit code for CUDA errors (gsamp_cuda.cu:23)
    }
    fprintf(stderr, "gsb2: %s\n", gsb_last_error());
    return rc;
}

static bool read_lines(const char *path, std::vector<std::string> &out) {
    FILE *g = fopen(path, "r");
    if (!g) return false;
    char line[4096];
    while (fgets(line, sizeof line, g)) out.push_back(line);
    fclose(g);
    return true;
}

static void put_bits(const int8_t *b, int ns) {
    for (int k = 0; k < ns; k++) putchar('0' + b[k]);
}

int main(int argc, char **argv) {
    if (argc < 4) return 1;
    int prec = 64;
    const char *pe = getenv("GSB_PRECISION");
    if (pe && atoi(pe) == 128) prec = 128;
    const size_t al = strlen(argv[0]);
    if (al >= 5 && !strcmp(argv[0] + al - 5, "_c128")) prec = 128;
    const int dev = getenv("GSB_DEVICE") ? atoi(getenv("GSB_DEVICE")) : 0;
    const int batch = getenv("GSB_BATCH") ? std::max(1, atoi(getenv("GSB_BATCH"))) : 64;

    gsb_engine *E = nullptr;
    int rc = gsb_open_file(argv[1], prec, dev, &E);
    if (rc) return die(rc);
    int n = 0, ns = 0, R = 0;
    gsb_info(E, &n, &ns, &R, nullptr);
    const char *mode = argv[2];

    if (!strcmp(mode, "sample") || !strcmp(mode, "sample2")) {
        const long N = atol(argv[3]);
        const unsigned long long seed = argc > 4 ? strtoull(argv[4], 0, 10) : 0;
        const int seeding = !strcmp(mode, "sample2") ? GSB_SEED_SEQ : GSB_SEED_INT;
        std::vector<int8_t> bits((size_t)batch * (size_t)std::max(ns, 1));
        std::vector<double> lp((size_t)batch);
        for (long i0 = 0; i0 < N; i0 += batch) {
            const long nb = std::min<long>(batch, N - i0);
            rc = gsb_sample(E, seeding, seed, i0, nb, bits.data(), lp.data());
            if (rc) return die(rc);
            for (long i = 0; i < nb; i++) {
                put_bits(bits.data() + i * ns, ns);
                printf(" %.12f %llu\n", lp[(size_t)i], seed + (unsigned long long)(i0 + i));
            }
            fflush(stdout);
        }
    } else if (!strcmp(mode, "prefix")) {
        if (argc < 6) return 1;
        const int K = atoi(argv[4]);
        const char *outp = argv[5];
        std::vector<std::string> lines;
        if (!read_lines(argv[3], lines)) return 1;
        int nk = 0, ntq = 1;
        gsb_dump_shape(E, K, &nk, &ntq);
        const size_t esz = prec == 128 ? 16 : 8, nent = ((size_t)1 << nk) * (size_t)ntq;
        std::vector<char> dump(nent * esz);
        std::vector<int8_t> fb((size_t)std::max(ns, 1));
        long li = 0;
        for (const std::string &line : lines) {
            if ((int)line.size() < K) continue;
            std::fill(fb.begin(), fb.end(), 0);
            for (int k = 0; k < K && k < ns; k++) {
                if (line[(size_t)k] == '?') { fprintf(stderr, "'?' before K in prefix mode\n"); return 8; }
                fb[(size_t)k] = (int8_t)(line[(size_t)k] - '0');
            }
            double logscale = 0, lp = 0;
            rc = gsb_prefix(E, fb.data(), K, dump.data(), &logscale, &lp);
            if (rc) return die(rc);
            char fn[1024];
            snprintf(fn, sizeof fn, "%s_%ld.bin", outp, li++);
            FILE *o = fopen(fn, "wb");
            if (!o) { fprintf(stderr, "cannot write %s\n", fn); return 1; }
            fwrite(&nk, 4, 1, o);
            fwrite(&ntq, 4, 1, o);
            fwrite(&logscale, 8, 1, o);
            fwrite(dump.data(), 1, dump.size(), o);
            fclose(o);
            printf("%ld %.12f %.6f\n", li - 1, lp, logscale);
            fflush(stdout);
        }
    } else if (!strcmp(mode, "resume")) {
        if (argc < 7) return 1;
        int nsl = argc - 6;
        const char *twistf = nullptr;
        if (argc >= 8 && !strcmp(argv[argc - 2], "--twist")) { twistf = argv[argc - 1]; nsl -= 2; }
        const int K = atoi(argv[4]);
        const unsigned long long seed = strtoull(argv[5], 0, 10);
        std::vector<std::string> lines;
        if (!read_lines(argv[3], lines)) return 1;
        int nk = 0, ntq = 1;
        gsb_dump_shape(E, K, &nk, &ntq);
        const size_t esz = prec == 128 ? 16 : 8, nent = ((size_t)1 << nk) * (size_t)ntq;
        std::vector<uint64_t> cs((size_t)nsl, 0), tqs((size_t)nsl, 0);
        if (twistf) {
            FILE *tf = fopen(twistf, "r");
            if (!tf) { fprintf(stderr, "missing twist file\n"); return 12; }
            for (int s = 0; s < nsl; s++) {
                unsigned long long a, b;
                if (fscanf(tf, "%llu %llu", &a, &b) != 2) { fprintf(stderr, "bad twist line %d\n", s); return 13; }
                cs[(size_t)s] = a;
                tqs[(size_t)s] = b;
            }
            fclose(tf);
        }
        std::vector<std::vector<char>> tabs((size_t)nsl, std::vector<char>(nent * esz));
        std::vector<const void *> ptr((size_t)nsl);
        std::vector<double> ls((size_t)nsl);
        std::vector<int8_t> fb((size_t)std::max(ns, 1)), bits((size_t)std::max(ns, 1));
        std::vector<double> cond((size_t)std::max(ns, 1));
        long li = 0;
        for (const std::string &line : lines) {
            if ((int)line.size() < ns) continue;
            for (int k = 0; k < ns; k++) fb[(size_t)k] = line[(size_t)k] == '?' ? -1 : (int8_t)(line[(size_t)k] - '0');
            for (int s = 0; s < nsl; s++) {
                char fn[1024];
                snprintf(fn, sizeof fn, "%s_%ld.bin", argv[6 + s], li);
                FILE *o = fopen(fn, "rb");
                if (!o) { fprintf(stderr, "missing %s\n", fn); return 9; }
                int nk2, ntq2;
                if (fread(&nk2, 4, 1, o) != 1 || nk2 != nk || fread(&ntq2, 4, 1, o) != 1 || ntq2 != ntq ||
                    fread(&ls[(size_t)s], 8, 1, o) != 1 || fread(tabs[(size_t)s].data(), esz, nent, o) != nent) {
                    fprintf(stderr, "bad dump %s\n", fn);
                    fclose(o);
                    return 10;
                }
                fclose(o);
                ptr[(size_t)s] = tabs[(size_t)s].data();
            }
            double lpf = 0, lpp = 0;
            rc = gsb_resume(E, fb.data(), K, seed, li, nsl, ptr.data(), ls.data(), twistf ? cs.data() : nullptr,
                            twistf ? tqs.data() : nullptr, bits.data(), &lpf, &lpp, cond.data());
            if (rc) return die(rc);
            put_bits(bits.data(), ns);
            printf(" %.12f %.12f", lpf, lpp);
            for (int k = K; k < ns; k++) printf(" %.9f", cond[(size_t)k]);
            putchar('\n');
            fflush(stdout);
            li++;
        }
    } else {
        // prob / chain / hybrid: lines of ns characters in step order
        const bool hybrid = !strcmp(mode, "hybrid"), ch = !strcmp(mode, "chain");
        const unsigned long long seed = hybrid && argc > 4 ? strtoull(argv[4], 0, 10) : 0;
        std::vector<std::string> all, lines;
        if (!read_lines(argv[3], all)) return 1;
        for (auto &l : all)
            if ((int)l.size() >= ns) lines.push_back(l);
        const size_t nsz = (size_t)std::max(ns, 1);
        std::vector<int8_t> fb((size_t)batch * nsz), bits((size_t)batch * nsz);
        std::vector<double> lp((size_t)batch), cond((size_t)batch * nsz);
        for (size_t i0 = 0; i0 < lines.size(); i0 += (size_t)batch) {
            const size_t nb = std::min(lines.size() - i0, (size_t)batch);
            for (size_t i = 0; i < nb; i++)
                for (int k = 0; k < ns; k++) {
                    const char c = lines[i0 + i][(size_t)k];
                    fb[i * nsz + (size_t)k] = hybrid && c == '?' ? -1 : (int8_t)(c - '0');
                }
            if (hybrid) rc = gsb_hybrid(E, fb.data(), (int64_t)nb, seed, (int64_t)i0, bits.data(), lp.data(), cond.data());
            else if (ch) rc = gsb_chain(E, fb.data(), (int64_t)nb, lp.data(), cond.data());
            else rc = gsb_prob(E, fb.data(), (int64_t)nb, lp.data());
            if (rc) return die(rc);
            for (size_t i = 0; i < nb; i++) {
                if (hybrid) {
                    put_bits(bits.data() + i * nsz, ns);
                    printf(" %.12f", lp[i]);
                    for (int k = 0; k < ns; k++) printf(" %.9f", cond[i * nsz + (size_t)k]);
                    putchar('\n');
                } else if (ch) {
                    printf("%.12f", lp[i]);
                    for (int k = 0; k < ns; k++) printf(" %.9f", cond[i * nsz + (size_t)k]);
                    putchar('\n');
                } else {
                    printf("%.12f\n", lp[i]);
                }
            }
            fflush(stdout);
        }
    }
    gsb_close(E);
    return 0;
}
