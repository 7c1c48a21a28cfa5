/*
 * testing_dpotrf_tlr -- command-line driver of the B200 TLR Cholesky.
 *
 * Same flags, phases and printed records as the reference driver
 * (hicma_parsec/testing_dpotrf.c:262-1107, options of hicma_parsec/hicma_parsec.c:89-309):
 * STARSH_gen -> rank statistics -> band auto-tuning + band regeneration ->
 * memory estimate -> HiCMA_dpotrf_L -> --check -> op counts -> R-LO line.
 * MPI/PaRSEC options (-P, -Q, -c, -g, the "--" MCA passthrough) are accepted
 * and ignored: one process drives one GPU.
 */
#define _GNU_SOURCE
#include <getopt.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "hicma_tlr.h"

static double wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static const char *str_problem[8] = {"randtlr", "ed-2d-sin", "st-2d-sqexp", "st-3d-sqexp",
                                     "st-3d-exp", "ed-3d-sin", "md-3d-virus", "md-3d-cube"};

/* Rank map block of tlr_rank_stat under PRINT_RANK (testing_dpotrf.c:91-106). */
static void print_rank_tile(const char *strid, const int *G, int NT, int band_size) {
    printf("%s %d %d\n", strid, NT, NT);
    for (int i = 0; i < NT; ++i) {
        for (int j = 0; j < NT; ++j) printf("%3d ", i - j >= band_size ? G[(size_t)j * NT + i] : -1);
        printf("\n");
    }
}

/* The five maps of parsec_rank_print (rank_print.jdf:128-183); tiles outside
 * the low-rank part print 0, as the reference's zero-initialised buffers do. */
static void print_rank_history(hicma_tlr_desc *A, int NT) {
    const size_t n2 = (size_t)NT * NT;
    int *h = malloc(sizeof(int) * n2 * 4);
    if (!h || hicma_tlr_rank_history(A, h, h + n2, h + 2 * n2, h + 3 * n2) != 0) { free(h); return; }
    static const char *title[5] = {"Initial Rank", "Minimum Rank", "Maximum Rank", "Final Rank",
                                   "Difference Rank, max - min"};
    for (int t = 0; t < 5; ++t) {
        printf("\n%s\n", title[t]);
        for (int i = 0; i < NT; ++i) {
            for (int j = 0; j < NT; ++j) {
                const size_t k = (size_t)j * NT + i;
                int v = t < 4 ? h[t * n2 + k] : h[2 * n2 + k] - h[n2 + k];
                if (h[k] < 0) v = 0;
                printf("%3d ", v);
            }
            printf("\n");
        }
        printf("\n\n");
    }
    free(h);
}

static void usage(void) {
    fprintf(stderr,
            "Mandatory: -N <n> -t <nb>\n"
            " -e --fixedacc     accuracy threshold (default 1e-8)\n"
            " -u --maxrank      storage maxrank (default NB/2)\n"
            " -G --genmaxrank   maxrank used in generation (default maxrank)\n"
            " -U --compmaxrank  maxrank of buffers (default maxrank)\n"
            " -f --fixedrank    fixed rank in recompression (0 = accuracy mode)\n"
            " -D --kind_of_problem 0: randtlr 1: ed-2d-sin 2: st-2d-sqexp 3: st-3d-sqexp 4: st-3d-exp 5: ed-3d-sin\n"
            "                      6: md-3d-virus 7: md-3d-cube\n"
            " -w --wavek        wave number of -D 1, 5 (default 50)\n"
            " -j --adddiag      diagonal of -D 0, 1, 5, 6, 7 (default N)\n"
            " -M --mesh_file    mesh of -D 6 (x y z per node)   -K --numobj  copies of it (default 1)\n"
            " -B --rbf_kernel   0 Gaussian 1 Expon 2 InvQUAD 3 InvMQUAD 4 Maternc1 5 Maternc2 6 TPS 7 CTPS 8 Wendland\n"
            " -R --radius       RBF shape radius (-D 6, 7; required)\n"
            " -O --order        0 none (default), 1 Morton   -S --density  packing of -D 6's copies (-1 random)\n"
            " -Z --band         band size (default 1)\n"
            " -E --auto-band    auto-tune band size (default 1)\n"
            " -Y --lookahead    lookahead (-1: band size)\n"
            " -F --send_full_tile, -W --two-flow, -z --HNB (accepted)\n"
            " -x --check        check against dense factorization\n"
            " -v --verbose\n"
            " --noise <nugget> (default 0.1, testing_dpotrf.c:305)  --beta <len> (0.1)\n"
            " --sigma <var> (1.0) --seed <s> (0) --precision fp64|mixed --ws <GiB> --device <id>\n"
            " --print-rank      print the rank maps (the reference's PRINT_RANK output)\n");
}

int main(int argc, char **argv) {
    int N = 0, NB = 0, maxrank = 0, genmaxrank = 0, compmaxrank = 0, fixedrk = 0, kind = 2, band_size = 1;
    int auto_band = 1, lookahead = -1, send_full_tile = 0, two_flow = 0, HNB = 300, check = 0, verbose = 0;
    int device = 0, precision = HICMA_TLR_PREC_FP64, print_rank = 0;
    double tol = 1e-8, noise = 0.1, beta = 0.1, sigma = 1.0, ws_gib = 0.0, wave_k = 50.0, add_diag = 0.0;
    int rbf_kernel = 0, numobj = 1, order = 0;   /* the reference's zero-initialised iparam (testing_dpotrf.c:265) */
    double radius = 0.0, density = -1.0;
    const char *mesh_file = NULL;
    unsigned long long seed = 0;
    static struct option opts[] = {
        {"N", required_argument, 0, 'N'},          {"NB", required_argument, 0, 't'},
        {"t", required_argument, 0, 't'},          {"fixedacc", required_argument, 0, 'e'},
        {"e", required_argument, 0, 'e'},          {"maxrank", required_argument, 0, 'u'},
        {"u", required_argument, 0, 'u'},          {"genmaxrank", required_argument, 0, 'G'},
        {"G", required_argument, 0, 'G'},          {"compmaxrank", required_argument, 0, 'U'},
        {"U", required_argument, 0, 'U'},          {"fixedrank", required_argument, 0, 'f'},
        {"f", required_argument, 0, 'f'},          {"kind_of_problem", required_argument, 0, 'D'},
        {"D", required_argument, 0, 'D'},          {"band", required_argument, 0, 'Z'},
        {"Z", required_argument, 0, 'Z'},          {"auto-band", required_argument, 0, 'E'},
        {"E", required_argument, 0, 'E'},          {"lookahead", required_argument, 0, 'Y'},
        {"Y", required_argument, 0, 'Y'},          {"send_full_tile", required_argument, 0, 'F'},
        {"F", required_argument, 0, 'F'},          {"two-flow", required_argument, 0, 'W'},
        {"W", required_argument, 0, 'W'},          {"HNB", required_argument, 0, 'z'},
        {"z", required_argument, 0, 'z'},          {"check", no_argument, 0, 'x'},
        {"x", no_argument, 0, 'x'},                {"verbose", optional_argument, 0, 'v'},
        {"v", optional_argument, 0, 'v'},          {"help", no_argument, 0, 'h'},
        {"h", no_argument, 0, 'h'},                {"P", required_argument, 0, 'P'},
        {"Q", required_argument, 0, 'Q'},          {"c", required_argument, 0, 'c'},
        {"cores", required_argument, 0, 'c'},      {"g", required_argument, 0, 'g'},
        {"wave_k", required_argument, 0, 'w'},     {"w", required_argument, 0, 'w'},
        {"wavek", required_argument, 0, 'w'},      {"adddiag", required_argument, 0, 'j'},
        {"add_diag", required_argument, 0, 'j'},   {"j", required_argument, 0, 'j'},
        {"grid-rows", required_argument, 0, 'P'},  {"grid-cols", required_argument, 0, 'Q'},
        /* RBF mesh problems (-D 6, 7, hicma_parsec.c:78-83) */
        {"rbf_kernel", required_argument, 0, 'B'}, {"B", required_argument, 0, 'B'},
        {"numobj", required_argument, 0, 'K'},     {"K", required_argument, 0, 'K'},
        {"mesh_file", required_argument, 0, 'M'},  {"M", required_argument, 0, 'M'},
        {"order", required_argument, 0, 'O'},      {"O", required_argument, 0, 'O'},
        {"radius", required_argument, 0, 'R'},     {"R", required_argument, 0, 'R'},
        {"density", required_argument, 0, 'S'},    {"S", required_argument, 0, 'S'},
        {"noise", required_argument, 0, 1001},     {"beta", required_argument, 0, 1002},
        {"sigma", required_argument, 0, 1003},     {"seed", required_argument, 0, 1004},
        {"precision", required_argument, 0, 1005}, {"ws", required_argument, 0, 1006},
        {"device", required_argument, 0, 1007},    {"print-rank", no_argument, 0, 1008},
        {0, 0, 0, 0}};
    int c, oi;
    while ((c = getopt_long_only(argc, argv, "", opts, &oi)) != -1) {
        switch (c) {
            case 'N': N = atoi(optarg); break;
            case 't': NB = atoi(optarg); break;
            case 'e': tol = atof(optarg); break;
            case 'u': maxrank = atoi(optarg); break;
            case 'G': genmaxrank = atoi(optarg); break;
            case 'U': compmaxrank = atoi(optarg); break;
            case 'f': fixedrk = atoi(optarg); break;
            case 'D': kind = atoi(optarg); break;
            case 'Z': band_size = atoi(optarg); break;
            case 'E': auto_band = atoi(optarg); break;
            case 'Y': lookahead = atoi(optarg); break;
            case 'F': send_full_tile = atoi(optarg); break;
            case 'W': two_flow = atoi(optarg); break;
            case 'z': HNB = atoi(optarg); break;
            case 'x': check = 1; verbose = 1; break;
            case 'v': verbose = optarg ? atoi(optarg) : 1; break;
            case 'h': usage(); return 0;
            case 'P': case 'Q': case 'c': case 'g': break;
            case 'B': rbf_kernel = atoi(optarg); break;
            case 'K': numobj = atoi(optarg); break;
            case 'M': mesh_file = optarg; break;
            case 'O': order = atoi(optarg); break;
            case 'R': radius = atof(optarg); break;
            case 'S': density = atof(optarg); break;
            case 'w': wave_k = atof(optarg); break;
            case 'j': add_diag = atof(optarg); break;
            case 1001: noise = atof(optarg); break;
            case 1002: beta = atof(optarg); break;
            case 1003: sigma = atof(optarg); break;
            case 1004: seed = strtoull(optarg, NULL, 10); break;
            case 1005: precision = strcmp(optarg, "mixed") == 0 ? HICMA_TLR_PREC_MIXED : HICMA_TLR_PREC_FP64; break;
            case 1006: ws_gib = atof(optarg); break;
            case 1007: device = atoi(optarg); break;
            case 1008: print_rank = 1; break;
            default: usage(); return 1;
        }
    }
    if (N <= 0 || NB <= 0) { fprintf(stderr, "#XXXXX the matrix size (N) and tile size (NB) are required\n"); usage(); return 1; }
    if (maxrank <= 0) { maxrank = NB / 2; fprintf(stderr, "Max rank has not been specified. Forced to the size of a tile %d\n", maxrank); }
    if (genmaxrank <= 0) genmaxrank = maxrank;
    if (compmaxrank <= 0) compmaxrank = maxrank;
    if (add_diag <= 0.0) add_diag = (double)N;   /* hicma_parsec.c:289-291 */
    if (kind < 0 || kind > 7) { fprintf(stderr, "Wrong value of \"kind_of_problem\" parameter\n"); return 1; }
    if (kind == 6 && !mesh_file) { fprintf(stderr, "-D 6 needs a mesh file (-M)\n"); return 1; }
    if ((kind == 6 || kind == 7) && !(radius > 0.0)) { fprintf(stderr, "-D 6, 7 need a positive radius (-R)\n"); return 1; }
    if (N % NB != 0) { fprintf(stderr, "N must be a multiple of NB\n"); return 1; }
    const int NT = N / NB;
    const double flops = (N * (((1. / 6.) * N + 0.5) * N + (1. / 3.))) + (N * (((1. / 6.) * N) * N - (1. / 6.)));
    if (verbose) {
        printf("M:%d N:%d NB:%d NB:%d HNB:%d HNB:%d\n", N, N, NB, NB, HNB, HNB);
        printf("kind_of_problem:%d %s\n", kind, str_problem[kind]);
        printf("tol:%.1e add_diag:%g fixed_rk:%d wave_k:%g\n", tol, add_diag, fixedrk, wave_k);
        if (kind == 6 || kind == 7)   /* testing_dpotrf.c:368 */
            printf("\nRBF, %s, %d, %d, %d, %d, %f, %f\n", mesh_file ? mesh_file : "(null)", N, rbf_kernel, numobj,
                   order, radius, density);
        printf("noise:%g beta:%g sigma:%g seed:%llu\n", noise, beta, sigma, seed);
        printf("send_full_tile:%d lookahead: %d band_size:%d max_rank:%d gen:%d comp:%d\n", send_full_tile,
               lookahead, band_size, maxrank, genmaxrank, compmaxrank);
    }
    if (auto_band) band_size = 1;   /* testing_dpotrf.c:407-414 */

    hicma_tlr_ctx *ctx = NULL;
    int rc = hicma_tlr_init(device, (size_t)(ws_gib * (1ull << 30)), &ctx);
    if (rc) { fprintf(stderr, "init failed: %s\n", hicma_tlr_last_error()); return 1; }
    hicma_tlr_set_precision(ctx, precision);
    hicma_tlr_problem prob = {kind, beta, 0.5, noise, sigma, seed, wave_k, add_diag,
                              rbf_kernel, radius, numobj, order, density};
    double *mesh_pts = NULL;   /* -D 6: the population of mesh copies */
    if (kind == 6) {
        mesh_pts = malloc(sizeof(double) * 3 * (size_t)N);
        rc = hicma_tlr_points_mesh(&prob, mesh_file, N, mesh_pts);
        if (rc) { fprintf(stderr, "mesh: %s\n", hicma_tlr_last_error()); return 1; }
    }
    hicma_tlr_desc *A = NULL;
    const int band_created = band_size;   /* slots of the off-band tiles are laid out for this band */
    rc = hicma_tlr_desc_create(ctx, N, NB, maxrank > genmaxrank ? maxrank : genmaxrank, band_size, &A);
    if (rc) { fprintf(stderr, "descriptor: %s\n", hicma_tlr_last_error()); return 1; }

    int info = 0, ret = 0;
    int *rank_array = malloc(sizeof(int) * NT * NT);
    double t0 = wtime();
    rc = hicma_tlr_generate(ctx, HICMA_TLR_LOWER, A, rank_array, &prob, mesh_pts, tol, genmaxrank, band_size,
                            send_full_tile, &info);
    const double time_starsh = wtime() - t0;
    printf("[****] TIME(s) %12.5f : STARSH_gen\tPxQ=   1 1   NB= %4d N= %7d\n", time_starsh, NB, N);
    if (rc || info != 0) {
        printf("Error in low rank matrix generation, info:%d rc:%d %s\n", info, rc, hicma_tlr_last_error());
        return 1;
    }
    int iminrk, imaxrk;
    double iavgrk;
    hicma_tlr_rank_stat(rank_array, NT, band_size, &iminrk, &imaxrk, &iavgrk);
    printf("[****] TIME(s) %12.5f : Gather rank\tband_size= %d  NT= %4d avg= %lf min= %d max= %d\n", 0.0, band_size,
           NT, iavgrk, iminrk, imaxrk);
    if (print_rank) print_rank_tile("init_rank_tile", rank_array, NT, band_size);
    const int imin_before = iminrk, imax_before = imaxrk;
    const double iavg_before = iavgrk;
    double time_opt_band = 0.0, time_regenerate = 0.0;
    if (auto_band) {
        t0 = wtime();
        const int band_opt = hicma_tlr_band_autotune(rank_array, NT, NB, verbose > 1);
        time_opt_band = wtime() - t0;
        printf("[****] TIME(s) %12.5f : band_size_auto_tuning\tNB= %4d N= %7d maxrank= %d band_size_opt= %d\n",
               time_opt_band, NB, N, maxrank, band_opt);
        t0 = wtime();
        if (band_opt != 1) {
            band_size = band_opt;
            rc = hicma_tlr_band_regenerate(ctx, HICMA_TLR_LOWER, A, &prob, band_size);
            if (rc) { fprintf(stderr, "band regeneration: %s\n", hicma_tlr_last_error()); return 1; }
        }
        time_regenerate = wtime() - t0;
        printf("[****] TIME(s) %12.5f : band_regeneration\tNB= %4d N= %7d band_size= %d\n", time_regenerate, NB, N,
               band_size);
        hicma_tlr_rank_gather(ctx, A, rank_array, band_size);
        hicma_tlr_rank_stat(rank_array, NT, band_size, &iminrk, &imaxrk, &iavgrk);
        if (print_rank) print_rank_tile("init_rank_tile", rank_array, NT, band_size);
    }
    /* memory estimate (testing_dpotrf.c:598-599) */
    const double mem = ((double)(NT - band_size) * (NT - band_size + 1) * NB * iavgrk + (double)band_size * NT * NB * NB) * 8 / 1073741824.0;
    const double mem_max = ((double)(NT - band_size) * (NT - band_size + 1) * NB * maxrank + (double)band_size * NT * NB * NB) * 8 / 1073741824.0;
    printf("[****] TIME(s) %12.5f : Memory_count\tNB= %4d N= %7d maxrank= %d band_size= %d memory_per_node= %lf GB memory_per_node_max= %lf GB\n",
           0.0, NB, N, maxrank, band_size, mem, mem_max);

    /* the matrix before factorization, for check_diff (testing_dpotrf.c:642-660) */
    hicma_tlr_desc *A0 = NULL;
    if (check) {
        rc = hicma_tlr_desc_create(ctx, N, NB, maxrank > genmaxrank ? maxrank : genmaxrank, band_created, &A0);
        if (rc == 0) rc = hicma_tlr_desc_copy(ctx, A, A0);
        if (rc) { fprintf(stderr, "copy for the check: %s\n", hicma_tlr_last_error()); return 1; }
    }
    unsigned long *tileops = calloc((size_t)NT * NT, sizeof(unsigned long));
    unsigned long opcounters[1] = {0};
    double cpt[6] = {0};
    t0 = wtime();
    info = hicma_tlr_dpotrf_L(ctx, HICMA_TLR_LOWER, A, rank_array, tol, fixedrk, maxrank, &lookahead, band_size, HNB,
                              compmaxrank, send_full_tile, &two_flow, tileops, opcounters, cpt, verbose);
    const double time_hicma = wtime() - t0;
    printf("[****] TIME(s) %12.5f : HiCMA_potrf\tsend_full_tile= %d band_size= %d lookahead= %d kind_of_problem= %d "
           "HNB= %d PxQ=   1 1   NB= %4d N= %7d 2flow= %d : %14f gflops\n",
           time_hicma, send_full_tile, band_size, lookahead, kind, HNB, NB, N, two_flow, flops / 1e9 / time_hicma);
    if (info < 0) { fprintf(stderr, "HiCMA_dpotrf_L error %d: %s\n", info, hicma_tlr_last_error()); return 1; }
    if (info != 0) { printf("-- Factorization is suspicious (info = %d) ! \n", info); ret |= 1; }
    if (print_rank) print_rank_history(A, NT);

    if (check && info == 0) {
        double res = 0, diff = 0;
        rc = hicma_tlr_check(ctx, A, &prob, A0, &res, &diff);
        if (rc) {
            fprintf(stderr, "check failed: %s\n", hicma_tlr_last_error());
            ret |= 1;
        } else {
            printf("Checking HiCMA L vs dense L: ||L-L0||_oo/||L||_oo = %e (threshold %.1e)\n", diff, tol);
            printf("-- %s\n", diff > tol || isnan(diff) ? "DIFFERENT matrices !" : "SAME matrices !");
            printf("Checking the Cholesky factorization. Threshold is %.2e\n", tol);
            printf("-- ||L'L-A||_oo/(||A||_oo) = %e\n", res);
            printf("-- Factorization is %s\n", res > tol || isnan(res) ? "suspicious !" : "CORRECT !");
            if (diff > tol || isnan(diff)) ret |= 1;
            if (res > tol || isnan(res)) ret |= 1;
            double ld = 0;
            hicma_tlr_logdet(ctx, A, &ld);
            printf("-- log det(A) = %.15e\n", ld);
        }
    }
    int fminrk, fmaxrk;
    double favgrk;
    hicma_tlr_rank_gather(ctx, A, rank_array, band_size);
    hicma_tlr_rank_stat(rank_array, NT, band_size, &fminrk, &fmaxrk, &favgrk);
    if (print_rank) print_rank_tile("rank_tile", rank_array, NT, band_size);
    unsigned long total = 0, band_ops = 0, offband_ops = 0;
    for (int i = 0; i < NT; ++i)
        for (int j = 0; j <= i; ++j) {
            total += tileops[(size_t)i * NT + j];
            if (i - j < band_size) band_ops += tileops[(size_t)i * NT + j];
            else offband_ops += tileops[(size_t)i * NT + j];
        }
    double st[12] = {0};
    hicma_tlr_last_stats(A, st, 12);
    const double path_ops = st[10], offpath_ops = (double)total - st[10];
    printf("[****] TIME(s) %12.5f : Operation_counts : band_size= %d total= %le op_band= %le op_offband= %le "
           "ratio_band= %lf op_critical_path= %le op_off_critical_path= %le ratio_critical_path= %lf\n",
           0.0, band_size, (double)total, (double)band_ops, (double)offband_ops,
           (double)band_ops / (double)offband_ops, path_ops, offpath_ops, path_ops / offpath_ops);
    printf("R-LO %d %d %d %d   %d %d   %d %d %d %d   %d %s %.1e %g %d %g   %d %d %d %d %d %d %d %d   "
           "%g %d %d   %g %d %d   %g %d %d   %lf %lf   %lf %lf %lf %lf    %lf %lf %lf %lf %lf    "
           "%le %le %le %le %le %lf %lf %d  ",
           N, N, NB, NB, HNB, HNB, 1, 1, 1, 1, kind, str_problem[kind], tol, add_diag, fixedrk, wave_k, send_full_tile,
           band_size, lookahead, 0, auto_band, maxrank, genmaxrank, compmaxrank, iavg_before, imin_before,
           imax_before, iavgrk, iminrk, imaxrk, favgrk, fminrk, fmaxrk, mem, mem_max, cpt[0] + cpt[1] + cpt[2],
           cpt[0], cpt[1], cpt[2], time_starsh, time_hicma, time_opt_band, time_regenerate, 0.0, (double)total,
           (double)band_ops, (double)offband_ops, path_ops, offpath_ops, (double)band_ops / (double)offband_ops,
           path_ops / offpath_ops, two_flow);
    if (kind == 6 || kind == 7) {   /* testing_dpotrf.c:1044-1047 */
        printf("%d %d %d  ", order, numobj, rbf_kernel);
        printf("%g %g ", radius, density);
    }
    printf("GITHASH:N/A    \"");
    for (int i = 0; i < argc; ++i) printf("%s ", argv[i]);
    printf("\"\n");
    free(tileops);
    free(rank_array);
    free(mesh_pts);
    if (A0) hicma_tlr_desc_destroy(A0);
    hicma_tlr_desc_destroy(A);
    hicma_tlr_fini(ctx);
    return ret;
}
