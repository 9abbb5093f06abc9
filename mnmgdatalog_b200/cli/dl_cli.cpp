// Command-line programs with the reference's interface, on libmnmgdl:
//
//   tc <file.bin> [cuda_aware] [method] [job_run]          tc.cu:78-95
//   sg <file.bin> [cuda_aware] [method] [job_run]          sg.cu:74-91
//   wcc <file.bin> [cuda_aware] [method] [job_run]         wcc.cu:97-113
//   single_join <rows> [cuda_aware] [method] [rand_range]  single_join.cu:81-100
//
// Same defaults, output file names (<input>_tc.bin, _sg.bin, _cc.bin,
// <rows>_singlejoin.bin) and CSV header/row as the reference programs (the
// MPI columns "Buffer preparation" and "Communication" are 0 on one GPU).
// cuda_aware and method select MPI strategies of the reference and are
// accepted and ignored. DL_WCC_STOP=fixpoint switches WCC to the true
// fixpoint stop rule. Build: python -m mnmgdatalog_b200.build (-DDL_CLI_PROGRAM=0..3).
#include <sys/stat.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mnmgdl.h"

#ifndef DL_CLI_PROGRAM
#define DL_CLI_PROGRAM 0
#endif

static void check(dl_status s, const char *what) {
    if (s != DL_OK) {
        fprintf(stderr, "GPUassert: %s: %s (%s)\n", what, dl_last_error(), dl_status_string(s));
        exit((int) s);
    }
}

static std::vector<int32_t> read_pairs(const char *path, int *rows_out) {
    // parallel_read (common/parallel_io.cu:5-41) with one rank: rows = size / 8
    struct stat st {};
    if (stat(path, &st) != 0) {
        printf("Error opening file %s", path);
        exit(EXIT_FAILURE);
    }
    const long long rows = (long long) st.st_size / 8;
    std::vector<int32_t> v((size_t) rows * 2);
    FILE *f = fopen(path, "rb");
    if (!f) {
        printf("Error opening file %s", path);
        exit(EXIT_FAILURE);
    }
    size_t got = rows ? fread(v.data(), 8, (size_t) rows, f) : 0;
    fclose(f);
    if ((long long) got != rows) {
        fprintf(stderr, "short read of %s\n", path);
        exit(EXIT_FAILURE);
    }
    *rows_out = (int) rows;
    return v;
}

static void write_pairs(const char *path, const std::vector<int32_t> &v) {
    FILE *f = fopen(path, "wb");
    if (!f) {
        fprintf(stderr, "cannot write %s\n", path);
        exit(EXIT_FAILURE);
    }
    if (!v.empty()) fwrite(v.data(), 4, v.size(), f);
    fclose(f);
}

int main(int argc, char **argv) {
    const int prog = DL_CLI_PROGRAM;
    const char *input = prog == DL_PROGRAM_WCC ? "data/dummy.bin" : "hipc_2019.bin";
    int job_run = prog == DL_PROGRAM_SINGLE_JOIN ? 1 : 0;
    int rand_range = 1000000;
    if (argc >= 2) input = argv[1];
    if (argc == 5) {
        if (prog == DL_PROGRAM_SINGLE_JOIN) rand_range = atoi(argv[4]);
        else job_run = atoi(argv[4]);
    }
    static const char *suffix[] = {"_tc.bin", "_sg.bin", "_cc.bin", "_singlejoin.bin"};
    const std::string out_name = std::string(input) + suffix[prog];

    double file_io = 0;
    int rows = 0;
    std::vector<int32_t> pairs;
    if (prog == DL_PROGRAM_SINGLE_JOIN) {
        rows = atoi(input);  // single_join.cu:100
        pairs.resize((size_t) rows * 2);
        check(dl_generate_rows(rows, rand_range, 1u, pairs.data()), "dl_generate_rows");
    } else {
        pairs = read_pairs(input, &rows);
    }

    dl_context *ctx = nullptr;
    check(dl_context_create(0, nullptr, &ctx), "dl_context_create");
    dl_options opt;
    memset(&opt, 0, sizeof(opt));
    opt.phase_timing = 1;
    const char *stop = getenv("DL_WCC_STOP");
    if (stop && std::string(stop) == "fixpoint") opt.wcc_stop = DL_WCC_STOP_FIXPOINT;
    dl_run *run = nullptr;
    check(dl_run_program(ctx, prog, pairs.data(), rows, 0, &opt, &run), "dl_run_program");
    dl_run_info info;
    check(dl_run_get_info(run, &info), "dl_run_get_info");
    std::vector<int32_t> out((size_t) info.output_rows * 2);
    check(dl_run_copy_output(run, out.data(), info.output_rows, 0), "dl_run_copy_output");
    if (job_run == 0) {
        write_pairs(out_name.c_str(), out);
        printf("Rank 0 wrote local tuples on file: %s\n", out_name.c_str());
    }
    const double init = info.seconds_init, join = info.seconds_join, dedup = info.seconds_dedup,
                 merge = info.seconds_merge, fin = info.seconds_finalize, total = info.seconds_total;
    if (prog == DL_PROGRAM_WCC) {
        printf("# Input,# Process,# Iterations,# CC,# Nodes in largest WCC,Total Time,Join,Buffer preparation,"
               "Communication,Deduplication,Merge,Initialization,Hashtable,Finalization,Clear,File I/O\n");
        printf("%d,%d,%d,%lld,%lld,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf\n", rows, 1,
               info.iterations, (long long) info.output_tuples, (long long) info.largest_component, total, join, 0.0,
               0.0, dedup, merge, init, 0.0, fin, 0.0, file_io);
    } else if (prog == DL_PROGRAM_SINGLE_JOIN) {
        printf("# Input,# Process,# Iterations,# Output,Total Time,Join,Buffer preparation (data distribution),"
               "Communication (data distribution),Buffer preparation (join result),Communication (join result),"
               "Deduplication,Clear,Copy,Finalization,Initialization,File I/O,Hashtable\n");
        printf("%d,%d,%d,%lld,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf\n", rows,
               1, info.iterations, (long long) info.output_tuples, total, join, 0.0, 0.0, 0.0, 0.0, dedup, 0.0, 0.0,
               fin, init, file_io, 0.0);
    } else {
        printf("# Input,# Process,# Iterations,# TC,Total Time,Join,Buffer preparation,Communication,"
               "Deduplication,Merge,Initialization,Hashtable,Finalization,Clear,File I/O\n");
        printf("%d,%d,%d,%lld,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf,%.4lf\n", rows, 1,
               info.iterations, (long long) info.output_tuples, total, join, 0.0, 0.0, dedup, merge, init, 0.0, fin,
               0.0, file_io);
    }
    dl_run_destroy(run);
    dl_context_destroy(ctx);
    return 0;
}
