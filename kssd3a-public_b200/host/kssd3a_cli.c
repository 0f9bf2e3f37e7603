/*
 * kssd3a — drop-in `kssd3a ani` front end over libkssdgpu.
 *
 * Options, defaults, validation messages and exit codes follow the reference's
 * `ani` (src/command_ani_wrapper.c:74-638; usage errors exit 64 through argp);
 * the path dispatcher follows run_sketch_ani (:1082-1230), and every output path
 * keeps its reference semantics (which AF precision, which anicut comparison, which
 * ordering) while all shared-context counting runs on the GPU:
 *
 *   mem_eff index path          src/command_ani.c:494-692 (+ counting filters src/command_ani.h:577-621)
 *   indexed self full/triangle  src/command_ani.c:1657-1842
 *   direct self / rect matrix   src/command_ani.c:3209-3365
 *   one-query stream            src/command_ani.c:2110-2201,2490-2666
 *   multi-query stream          src/command_ani.c:2792-3015
 *   no-index hash detail        src/command_ani.c:3837-4000
 *
 * Inputs are sketch directories, or FASTA/FASTQ files and directories of them, which
 * are sketched on the GPU first (auto ANI, src/command_ani_wrapper.c:842-1046,1275-1502;
 * host/kssd_autosketch.c).
 */
#define _GNU_SOURCE
#include <argp.h>
#include <ctype.h>
#include <err.h>
#include <errno.h>
#include <fcntl.h>
#include <inttypes.h>
#include <limits.h>
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <pthread.h>
#include <unistd.h>

#include "kssd_epilogue.h"
#include "kssd_format.h"
#include "kssd_hgb.h"
#include "kssd_autosketch.h"
#include "kssd_fastx.h"
#include "kssdgpu.h"

#define PATHLEN KSSD_PATHLEN

const char *argp_program_version = "kssd3a (B200 counting engine) 3.2.0-rc.1";

typedef struct cli {
    kssd_ani_opt_t o;
    char refdir[PATHLEN], qrydir[PATHLEN], outf[PATHLEN], unique_report[PATHLEN];
    char reflist[PATHLEN], qrylist[PATHLEN], gl[PATHLEN], index[PATHLEN], model[PATHLEN], pipecmd[PATHLEN];
    double c;
    bool pair, estimate_coverage, unique_ctx;
    int output_values, coden_seen, manual_seen;
    bool sketch_coden;
    int sketch_hclen, sketch_holen, sketch_iolen, sketch_drfold, sketch_kmerocrs, sketch_ncap;
    double sketch_npercentile;
    bool sketch_split_mfa, sketch_abundance, sketch_anno, sketch_conflict, sketch_asone, sketch_reads_qc;
    int nrem;
    char **rem;
} cli_t;

static cli_t g;

/* ------------------------------------------------------------------ options */

enum {
    O_USE_CODEN = 781, O_CTXLEN, O_OUTEROBJLEN, O_INNEROBJLEN, O_DRFOLD, O_LSTKMER, O_NPERCENTILE, O_NCAP,
    O_READSQC, O_ABUNDANCE, O_ANNO, O_CONFLICT, O_ASONE, O_SPLITMFA, O_PIPECMD, O_RAW_OUTPUT, O_UNIFIED,
    O_COVERAGE, O_MAX_PDIST, O_MAX_DIFF, O_METRIC, O_FORMAT, O_VALUES, O_UNIQUE_REPORT, O_UNIQUE
};

static struct argp_option k_opts[] = {
    {0, 0, 0, 0, "Input sketches:", 1},
    {"ref", 'r', "<SKETCH>", 0, "Reference sketch directory.", 1},
    {"query", 'q', "<SKETCH>", 0, "Query sketch directory.", 1},
    {"qraw", 'x', "<SKETCH>", 0, "Raw-read query sketch directory; enables naive ANI mode.", 1},
    {"reflist", 779, "<FILE>", 0, "Reference FASTA/FASTQ/sketch path list for auto ANI.", 1},
    {"qrylist", 780, "<FILE>", 0, "Query FASTA/FASTQ/sketch path list for auto ANI.", 1},
    {"index", 'i', "<FILE>", OPTION_HIDDEN, "Reserved; currently unused.", 2},
    {0, 0, 0, 0, "ANI mode and conflict handling:", 2},
    {"naive", 'v', 0, 0, "Use naive distance/ANI calculation.", 2},
    {"ignoreconflict", 778, 0, 0, "Ignore reference-side contexts that contain conflicting objects.", 2},
    {"unique-ctx", O_UNIQUE, 0, 0, "Adaptive read-to-reference naive ANI on reference-unique contexts "
                                  "(>= 5% of full reference contexts); indexed -r and --qraw, detail only.", 2},
    {0, 0, 0, 0, "Filtering and metrics:", 3},
    {"afcut", 'f', "<0..1>", 0, "Skip reports with max(Qry_align_fraction, Ref_align_fraction) below this fraction. [0.5; 0.2 for --qraw]", 3},
    {"anicut", 'n', "<0..1>", 0, "Skip reports with ANI below this fraction. [0.95]", 3},
    {"metric", O_METRIC, "<NAME>", 0, "best, recalibrated, ctx-moe, ctx-naive, p_dist, mash, aaf, mash-if-far, aaf-if-far. [best]", 3},
    {"control", 'c', "<FLOAT>", 0, "Skip duplicated samples with distance below this value. [0]", 3},
    {"ctxcut", 't', "<INT>", 0, "Skip reports with overlapped context count below this value. [3]", 3},
    {"slmetrics", 's', "<+-1..9>", 0, "Metric number 1..9; in matrix mode positive reports distance, negative ANI. [1]", 3},
    {"max-pdist", O_MAX_PDIST, "<FLOAT>", 0, "Close-only detail filter on p_dist. [off]", 3},
    {"max-diff-section", O_MAX_DIFF, "<INT>", 0, "Close-only detail filter on object-section differences. [off]", 3},
    {"unified-metric", O_UNIFIED, 0, 0, "In --qraw mode honor -s instead of forcing Naive.", 3},
    {0, 0, 0, 0, "Reporting and output:", 4},
    {"diagonal", 'd', 0, 0, "Set diagonal values.", 4},
    {"exception", 'e', "<INT>", 0, "Missing/low-overlap matrix distance [1]; ANI uses 1-e.", 4},
    {"glist", 'g', "<FILE>", 0, "Sample output file for KSSD set grouping.", 4},
    {"outfmt", 'm', "<0/1/2>", 0, "Output format: detail(0), matrix(1), or triangle(2). [0]", 4},
    {"format", O_FORMAT, "<NAME>", 0, "detail, matrix, or triangle; alias for -m. [detail]", 4},
    {"values", O_VALUES, "<distance|ani>", 0, "Matrix/triangle values; overrides the sign of -s. [distance]", 4},
    {"outfile", 'o', "<FILE>", 0, "Output file. [STDOUT]", 4},
    {"raw-output", O_RAW_OUTPUT, 0, 0, "Skip calibrated/best ANI computation.", 4},
    {"estimate-coverage", O_COVERAGE, 0, 0,
     "Append abundance-derived coverage/depth columns for --qraw detail output when the query sketch has comblco.a.",
     4},
    {"unique-ctx-report", O_UNIQUE_REPORT, "<FILE>", 0, "Write unfiltered unique-context counts to a new file.", 4},
    {"top", 'N', "<INT>", 0, "Report at most top N references per query. [all]", 4},
    {0, 0, 0, 0, "Execution:", 5},
    {"threads", 'p', "<INT>", 0, "Number of host threads for the epilogue.", 5},
    {0, 0, 0, 0, "Direct FASTA/FASTQ input mode:", 6},
    {"pair", 777, 0, 0, "Treat positional inputs as reference then query inputs.", 6},
    {"pipecmd", O_PIPECMD, "<cmd>", 0, "Stream each raw input through command.", 6},
    {"use_coden_ctxobj", O_USE_CODEN, 0, 0, "Use the coden context-object pattern. [default]", 7},
    {"DimRdcFold", O_DRFOLD, "<INT>", 0, "K-mer space downsampling rate 1/2^f. [8]", 7},
    {"ctxlen", O_CTXLEN, "<INT>", 0, "Manual half context length.", 7},
    {"outerobjlen", O_OUTEROBJLEN, "<INT>", 0, "Manual half outer object length.", 7},
    {"innerobjlen", O_INNEROBJLEN, "<INT>", 0, "Manual inner object length.", 7},
    {"LstKmerOcrs", O_LSTKMER, "<INT>", 0, "Least k-mer occurrence required in FASTQ input. [1]", 7},
    {"npercentile", O_NPERCENTILE, "<0..1>", 0, "Weighted lower-tail count percentile.", 7},
    {"ncap", O_NCAP, "<INT>", OPTION_HIDDEN, "Cap for effective lower k-mer occurrence cutoff. [0]", 7},
    {"readsQC", O_READSQC, 0, 0, "Infer and apply read-count QC filtering.", 7},
    {"abundance", O_ABUNDANCE, 0, 0, "Use abundance-estimation mode.", 7},
    {"anno", O_ANNO, 0, 0, "Write FASTA/FASTQ header annotations.", 7},
    {"conflict", O_CONFLICT, 0, 0, "Keep conflicting context-objects.", 7},
    {"asone", O_ASONE, 0, 0, "Treat each raw input path as one final genome.", 7},
    {"splitmfa", O_SPLITMFA, 0, 0, "Treat each multi-FASTA record as one genome.", 7},
    {0}};

static int parse_int_range(struct argp_state *st, const char *name, const char *arg, int lo, int hi)
{
    char *end = NULL;
    errno = 0;
    long v = strtol(arg, &end, 10);
    if (errno || end == arg || *end || v < lo || v > hi)
        argp_error(st, "%s requires an integer in range %d..%d", name, lo, hi);
    return (int)v;
}

static double parse_double_range(struct argp_state *st, const char *name, const char *arg, double lo, double hi)
{
    char *end = NULL;
    errno = 0;
    double v = strtod(arg, &end);
    if (errno || end == arg || *end || !isfinite(v) || v < lo || v > hi)
        argp_error(st, "%s requires a number in range %.6g..%.6g", name, lo, hi);
    return v;
}

static void copy_path(struct argp_state *st, const char *name, char *dst, const char *arg)
{
    if (strlen(arg) >= PATHLEN)
        argp_error(st, "%s path is too long; maximum supported length is %d bytes", name, PATHLEN - 1);
    snprintf(dst, PATHLEN, "%s", arg);
}

static error_t parse_ani(int key, char *arg, struct argp_state *st)
{
    kssd_ani_opt_t *o = &g.o;
    switch (key) {
    case O_UNIQUE: g.unique_ctx = o->unique_ctx = true; break;
    case O_UNIQUE_REPORT: copy_path(st, "--unique-ctx-report", g.unique_report, arg); break;
    case O_METRIC: {
        static const char *names[] = {"best", "recalibrated", "ctx-moe", "ctx-naive", "mash", "aaf",
                                      "mash-if-far", "aaf-if-far", "p_dist"};
        int m = 0;
        for (int i = 0; i < 9; ++i)
            if (!strcmp(arg, names[i]))
                m = i + 1;
        if (!strcmp(arg, "naive")) m = 4;
        if (!strcmp(arg, "pdist")) m = 9;
        if (!m)
            argp_error(st, "unknown --metric '%s'; use best, recalibrated, ctx-moe, ctx-naive, p_dist, mash, aaf, "
                           "mash-if-far, or aaf-if-far", arg);
        o->s = o->s < 0 ? -m : m;
        break;
    }
    case O_FORMAT:
        if (!strcmp(arg, "detail")) o->fmt = 0;
        else if (!strcmp(arg, "matrix")) o->fmt = 1;
        else if (!strcmp(arg, "triangle")) o->fmt = 2;
        else argp_error(st, "--format must be detail, matrix, or triangle");
        break;
    case O_VALUES:
        if (!strcmp(arg, "distance")) g.output_values = 1;
        else if (!strcmp(arg, "ani")) g.output_values = -1;
        else argp_error(st, "--values must be distance or ani");
        break;
    case 'm': o->fmt = parse_int_range(st, "-m/--outfmt", arg, 0, 2); break;
    case 'c': {
        char *end = NULL;
        errno = 0;
        double v = strtod(arg, &end);
        if (errno || end == arg || *end || !isfinite(v) || v < 0.0)
            argp_error(st, "%s requires a non-negative number", "-c/--control");
        g.c = v;
        break;
    }
    case 'e': o->e = parse_int_range(st, "-e/--exception", arg, 1, INT_MAX); break;
    case 's':
        o->s = parse_int_range(st, "-s/--slmetrics", arg, -9, 9);
        if (o->s == 0)
            argp_error(st, "-s/--slmetrics accepts -9..-1 or 1..9, but not 0");
        break;
    case 'p': o->p = parse_int_range(st, "-p/--threads", arg, 1, 65536); break;
    case O_USE_CODEN: g.coden_seen = 1; g.sketch_coden = true; break;
    case O_CTXLEN: g.manual_seen = 1; g.sketch_coden = false; g.sketch_hclen = parse_int_range(st, "--ctxlen", arg, 4, 16); break;
    case O_OUTEROBJLEN: g.manual_seen = 1; g.sketch_coden = false; g.sketch_holen = parse_int_range(st, "--outerobjlen", arg, 0, 8); break;
    case O_INNEROBJLEN: g.manual_seen = 1; g.sketch_coden = false; g.sketch_iolen = parse_int_range(st, "--innerobjlen", arg, 0, 8); break;
    case O_DRFOLD: g.sketch_drfold = parse_int_range(st, "--DimRdcFold", arg, 0, 24); break;
    case O_LSTKMER: g.sketch_kmerocrs = parse_int_range(st, "--LstKmerOcrs", arg, 1, 65536); break;
    case O_NPERCENTILE: g.sketch_npercentile = parse_double_range(st, "--npercentile", arg, 0.0, 1.0); break;
    case O_NCAP: g.sketch_ncap = parse_int_range(st, "--ncap", arg, 0, 65536); break;
    case O_READSQC:
        g.sketch_reads_qc = true;
        if (g.sketch_kmerocrs < 2)
            g.sketch_kmerocrs = 2;
        break;
    case O_ABUNDANCE: g.sketch_abundance = true; break;
    case O_ANNO: g.sketch_anno = true; break;
    case O_CONFLICT: g.sketch_conflict = true; break;
    case O_ASONE: g.sketch_asone = true; break;
    case O_SPLITMFA: g.sketch_split_mfa = true; break;
    case O_PIPECMD: copy_path(st, "--pipecmd", g.pipecmd, arg); break;
    case O_RAW_OUTPUT: o->raw_output = true; break;
    case O_UNIFIED: o->unified_metric = true; break;
    case O_COVERAGE: g.estimate_coverage = true; break;
    case O_MAX_PDIST: o->max_pdist = parse_double_range(st, "--max-pdist", arg, 0.0, 1.0); o->max_pdist_set = true; break;
    case O_MAX_DIFF: o->max_diff_obj_section = parse_int_range(st, "--max-diff-section", arg, 0, INT_MAX); break;
    case 't': o->ctxcut = parse_int_range(st, "-t/--ctxcut", arg, 0, INT_MAX); break;
    case 'f':
        o->afcut = (float)parse_double_range(st, "-f/--afcut (fraction, e.g. 0.8, not 80)", arg, 0.0, 1.0);
        o->afcut_set = true;
        break;
    case 'n': o->anicut = (float)parse_double_range(st, "-n/--anicut (fraction, e.g. 0.95, not 95)", arg, 0.0, 1.0); break;
    case 'N': o->ntop = parse_int_range(st, "-N/--top", arg, 1, INT_MAX); break;
    case 'i': copy_path(st, "-i/--index", g.index, arg); break;
    case 'M': copy_path(st, "-M/--model", g.model, arg); break;
    case 'q': copy_path(st, "-q/--query", g.qrydir, arg); break;
    case 780: copy_path(st, "--qrylist", g.qrylist, arg); break;
    case 'r': copy_path(st, "-r/--ref", g.refdir, arg); break;
    case 779: copy_path(st, "--reflist", g.reflist, arg); break;
    case 'o': copy_path(st, "-o/--outfile", g.outf, arg); break;
    case 'g': copy_path(st, "-g/--glist", g.gl, arg); break;
    case 'd': o->d = true; break;
    case 'v': o->v = true; break;
    case 778: o->ignoreconflict = true; break;
    case 'x':
        copy_path(st, "--qraw", g.qrydir, arg);
        o->unassembled = true;
        o->v = true;
        break;
    case 777: g.pair = true; break;
    case ARGP_KEY_ARGS:
        g.nrem = st->argc - st->next;
        g.rem = st->argv + st->next;
        break;
    case ARGP_KEY_END: {
        /* validation, src/command_ani_wrapper.c:536-621 */
        if (g.output_values)
            o->s = abs(o->s) * g.output_values;
        const bool has_reflist = g.reflist[0], has_qrylist = g.qrylist[0];
        if (g.unique_ctx || g.unique_report[0]) {
            if (!o->unassembled || o->fmt != 0 || !g.refdir[0] || !g.qrydir[0] || has_reflist || has_qrylist || g.nrem)
                argp_error(st, "unique-context options require explicit -r/--qraw inputs and detail output");
            if (g.unique_ctx && (o->unified_metric || o->raw_output || abs(o->s) > 4 || o->max_pdist_set ||
                                 o->max_diff_obj_section >= 0))
                argp_error(st, "--unique-ctx uses calibrated read-mode Naive ANI; incompatible metric, raw-output, "
                               "unified-metric or close-pair filter");
            if (g.unique_report[0] && !strcmp(g.unique_report, g.outf))
                argp_error(st, "--unique-ctx-report must differ from the ordinary output path");
        }
        if (g.coden_seen && g.manual_seen)
            argp_error(st, "--use_coden_ctxobj selects the coden pattern; do not combine it with --ctxlen, "
                           "--outerobjlen, or --innerobjlen.");
        if (!g.sketch_coden) {
            int k = g.sketch_iolen + 2 * (g.sketch_holen + g.sketch_hclen);
            if (k > 32)
                argp_error(st, "auto-sketch k-mer length %d should be at most 32", k);
        }
        if (g.pipecmd[0] && g.sketch_split_mfa)
            argp_error(st, "--splitmfa does not support --pipecmd streaming inputs");
        if (g.estimate_coverage && o->fmt != 0)
            argp_error(st, "--estimate-coverage is supported only with detail output (-m0).");
        if (g.estimate_coverage && !o->unassembled)
            argp_error(st, "--estimate-coverage currently requires --qraw raw/unassembled query mode.");
        if ((o->max_pdist_set || o->max_diff_obj_section >= 0) && o->fmt != 0)
            argp_error(st, "--max-pdist/--max-diff-section are supported only with detail output (-m0).");
        if (has_reflist || has_qrylist) {
            if (!has_reflist || !has_qrylist)
                argp_error(st, "--reflist and --qrylist must be used together");
            if (g.refdir[0] || g.qrydir[0])
                argp_error(st, "--reflist/--qrylist cannot be combined with -r, -q, or --qraw");
            if (g.pair || g.nrem > 0)
                argp_error(st, "--reflist/--qrylist cannot be combined with --pair or positional inputs");
        } else if (g.pair) {
            if (g.refdir[0] || g.qrydir[0])
                argp_error(st, "--pair cannot be combined with -r, -q, or --qraw");
            if (g.nrem < 2)
                argp_error(st, "--pair requires one reference input followed by at least one query input");
        } else if (!g.refdir[0] && !g.qrydir[0] && g.nrem >= 2) {
            g.pair = true;
        } else if (!g.refdir[0] && !g.qrydir[0] && g.nrem == 1 && o->fmt != 0) {
            copy_path(st, "sketch", g.qrydir, g.rem[0]);
        } else if (!g.qrydir[0]) {
            argp_error(st, "missing query: use -q, --qraw, or positional reference and query inputs");
        } else if (!g.refdir[0] && o->fmt == 0) {
            argp_error(st, "-r/--ref is required for detail output; use -m1 or -m2 for one-sketch self matrices");
        }
        if (o->s < -9 || o->s > 9 || o->s == 0)
            argp_error(st, "-s option should be within range 1..9 or -9..-1");
        break;
    }
    default:
        return ARGP_ERR_UNKNOWN;
    }
    return 0;
}

static struct argp k_argp = {
    k_opts, parse_ani,
    "[-r REF_SKETCH -q QRY | -r REF_SKETCH --qraw RAW_QRY | SELF_SKETCH with -m1/-m2]",
    "\nEstimate average nucleotide identity (ANI) between sketches; shared-context counting on the GPU."
    "\vOutputs are byte-identical to the reference `kssd3a ani` on the same sketch directories.",
    NULL, NULL, NULL};

/* ------------------------------------------------------------------ helpers */

static int env_int(const char *name, int dflt, int lo, const char *what)
{
    const char *e = getenv(name);
    if (!e || !e[0])
        return dflt;
    char *end = NULL;
    errno = 0;
    long v = strtol(e, &end, 10);
    if (errno || end == e || *end || v < lo || v > INT_MAX)
        errx(EXIT_FAILURE, "invalid %s='%s' (use %s)", name, e, what);
    return (int)v;
}

static bool force_ref_index(void)
{
    const char *e = getenv("KSSD3A_FORCE_REF_INDEX");
    return e && e[0] && strcmp(e, "0") != 0;
}

static int matrix_direct_threshold(void)
{
    const char *name = "KSSD3A_ANI_MATRIX_DIRECT_THRESHOLD";
    const char *e = getenv(name);
    if (!e || !e[0]) {
        name = "KSSD3A_ANI_M1_DIRECT_THRESHOLD";
        e = getenv(name);
    }
    if (!e || !e[0])
        return 1000;
    char *end = NULL;
    errno = 0;
    long v = strtol(e, &end, 10);
    if (errno || end == e || *end || v < 0 || v > INT_MAX)
        errx(EXIT_FAILURE, "invalid %s='%s' (use non-negative integer)", name, e);
    return (int)v;
}

static bool matrix_use_index(int nref, int nq, int direct)
{
    if (nref < 1 || nq < 1)
        return false;
    if (direct == 0)
        return true;
    return nref > direct || nq > direct;
}

static bool same_file(const char *a, const char *b)
{
    struct stat sa, sb;
    return a && b && !stat(a, &sa) && !stat(b, &sb) && sa.st_dev == sb.st_dev && sa.st_ino == sb.st_ino;
}

static bool is_sketch_dir(const char *p)
{
    struct stat st;
    if (stat(p, &st) || !S_ISDIR(st.st_mode))
        return false;
    return kssd_file_exists(p, "lcofiles.stat") && kssd_file_exists(p, "comblco") && kssd_file_exists(p, "comblco.index");
}

static kssd_sketch_t *load_sketch(const char *dir, unsigned flags)
{
    kssd_sketch_t *s = kssd_sketch_load(dir, flags);
    if (!s)
        errx(EXIT_FAILURE, "%s", kssd_host_last_error());
    return s;
}

static void gpu_check(int rc, const char *what)
{
    if (rc != KSSDGPU_OK)
        errx(EXIT_FAILURE, "%s: %s", what, kssdgpu_last_error());
}

/* CUDA context creation takes a sizeable fraction of a short run: start it on a
 * helper thread while the sketches and the index are read (the runtime makes a later
 * first call from the main thread wait for it). */
static void *gpu_warmup(void *arg)
{
    (void)arg;
    kssdgpu_init(0);
    return NULL;
}

static void start_gpu_warmup(void)
{
    pthread_t t;
    if (pthread_create(&t, NULL, gpu_warmup, NULL) == 0)
        pthread_detach(t);
}

static FILE *open_out(const char *path)
{
    FILE *f = path[0] ? fopen(path, "w") : stdout;
    if (!f)
        err(errno, "%s", path);
    return f;
}

static void close_out(FILE *f)
{
    if (fflush(f) != 0 || ferror(f))
        err(EXIT_FAILURE, "Cannot write ANI output");
    if (f != stdout && fclose(f) != 0)
        err(EXIT_FAILURE, "Cannot finish ANI output");
}

static void write_buf(FILE *f, const kssd_buf_t *b)
{
    if (b->l && fwrite(b->s, 1, b->l, f) != b->l)
        err(EXIT_FAILURE, "Cannot write ANI output");
}

/* Ordered background writer: chunks of formatted rows handed over in order are
 * written by one thread while the caller formats the next chunk (at most one chunk
 * queued behind the one being written). */
typedef struct {
    kssd_buf_t *rows;
    int nb;
} wchunk_t;

typedef struct {
    FILE *f;
    pthread_t th;
    pthread_mutex_t mu;
    pthread_cond_t cv;
    wchunk_t q[2];
    int head, count;
    bool done;
} owriter_t;

static void *owriter_main(void *arg)
{
    owriter_t *w = arg;
    for (;;) {
        pthread_mutex_lock(&w->mu);
        while (!w->count && !w->done)
            pthread_cond_wait(&w->cv, &w->mu);
        if (!w->count) {
            pthread_mutex_unlock(&w->mu);
            return NULL;
        }
        const wchunk_t c = w->q[w->head];
        pthread_mutex_unlock(&w->mu);
        for (int i = 0; i < c.nb; ++i) {
            write_buf(w->f, &c.rows[i]);
            kssd_buf_free(&c.rows[i]);
        }
        free(c.rows);
        pthread_mutex_lock(&w->mu);
        w->head = (w->head + 1) % 2;
        w->count--;
        pthread_cond_broadcast(&w->cv);
        pthread_mutex_unlock(&w->mu);
    }
}

static void owriter_start(owriter_t *w, FILE *f)
{
    memset(w, 0, sizeof *w);
    w->f = f;
    pthread_mutex_init(&w->mu, NULL);
    pthread_cond_init(&w->cv, NULL);
    if (pthread_create(&w->th, NULL, owriter_main, w) != 0)
        errx(EXIT_FAILURE, "cannot start the output writer thread");
}

static void owriter_push(owriter_t *w, kssd_buf_t *rows, int nb)
{
    pthread_mutex_lock(&w->mu);
    while (w->count == 2)
        pthread_cond_wait(&w->cv, &w->mu);
    w->q[(w->head + w->count) % 2] = (wchunk_t){rows, nb};
    w->count++;
    pthread_cond_broadcast(&w->cv);
    pthread_mutex_unlock(&w->mu);
}

static void owriter_finish(owriter_t *w)
{
    pthread_mutex_lock(&w->mu);
    w->done = true;
    pthread_cond_broadcast(&w->cv);
    pthread_mutex_unlock(&w->mu);
    pthread_join(w->th, NULL);
    pthread_mutex_destroy(&w->mu);
    pthread_cond_destroy(&w->cv);
}

/* KSSD3A_TIMING=1: phase timings on stderr */
static double g_t_last = -1.0;
static void phase(const char *what)
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("KSSD3A_TIMING");
        on = e && e[0] && strcmp(e, "0");
    }
    if (!on)
        return;
    const double now = omp_get_wtime();
    if (g_t_last >= 0)
        fprintf(stderr, "[kssd3a] %-28s %8.1f ms\n", what, 1e3 * (now - g_t_last));
    g_t_last = now;
}

/* context runs of one sorted sample (count_ctx_runs_sorted_ctxobj64_local, src/command_ani.c:337-349) */
static uint32_t ctx_runs(const uint64_t *a, size_t n, int obj_bits, bool ignoreconflict)
{
    uint32_t runs = 0;
    for (size_t i = 0; i < n;) {
        const uint64_t ctx = a[i] >> obj_bits;
        const size_t b = i;
        do {
            ++i;
        } while (i < n && (a[i] >> obj_bits) == ctx);
        if (!ignoreconflict || i - b == 1)
            runs++;
    }
    return runs;
}

static uint32_t *sample_ctx_counts(const kssd_sketch_t *s, bool use_runs, bool ignoreconflict)
{
    uint32_t *c = calloc((size_t)(s->n ? s->n : 1), sizeof(uint32_t));
    if (!c)
        err(EXIT_FAILURE, "calloc ctx counts");
#pragma omp parallel for schedule(dynamic, 64) num_threads(g.o.p)
    for (int i = 0; i < s->n; ++i) {
        const size_t len = (size_t)(s->offs[i + 1] - s->offs[i]);
        c[i] = use_runs ? ctx_runs(s->keys + s->offs[i] - s->offs[0], len, s->obj_bits, ignoreconflict) : (uint32_t)len;
    }
    return c;
}

static const char *anno_at(const kssd_sketch_t *s, uint32_t i)
{
    return s && s->anno && s->anno[i][0] ? s->anno[i] : "NA";
}

static bool best_guard_enabled(void) { return g.o.fmt == 0 && !g.o.unassembled && !g.o.v; }

static unsigned ref_flags(void) { return (g.o.fmt == 0 ? 1u : 0u) | (best_guard_enabled() ? 2u : 0u); }
static unsigned qry_flags(void) { return best_guard_enabled() ? 2u : 0u; }

static void init_bits(const kssd_sketch_t *q)
{
    g.o.drfold = q->stat.drfold;
    g.o.obj_bits = q->obj_bits;
    g.o.ctx_bits = q->ctx_bits;
}

static kssdgpu_index_t *gpu_index_of_sketch(const kssd_sketch_t *s)
{
    kssdgpu_index_t *ix = NULL;
    gpu_check(kssdgpu_index_from_sketch(s->keys, s->offs, s->n, s->obj_bits, 0, &ix), "device index");
    return ix;
}

/* Counters of queries [q0, q0+nb) against the index: [nb][R] cells each. */
typedef struct counts {
    kssdgpu_ctx_mut2_t *ctx, *uctx;
    kssdgpu_obj_section_t *obj, *uobj;
} counts_t;

static counts_t count_queries(kssdgpu_index_t *ix, int nref, const kssd_sketch_t *q, int q0, int nb, unsigned flags)
{
    counts_t c = {0};
    const size_t cells = (size_t)nb * (size_t)nref;
    c.ctx = malloc(cells * sizeof(*c.ctx) + 1);
    c.obj = malloc(cells * sizeof(*c.obj) + 1);
    if (flags & KSSDGPU_UNIQUE) {
        c.uctx = malloc(cells * sizeof(*c.uctx) + 1);
        c.uobj = malloc(cells * sizeof(*c.uobj) + 1);
    }
    if (!c.ctx || !c.obj || ((flags & KSSDGPU_UNIQUE) && (!c.uctx || !c.uobj)))
        err(EXIT_FAILURE, "OOM counter block");
    const uint64_t *keys = q->keys + (q->offs[q0] - q->offs[0]);
    gpu_check(kssdgpu_count_block(ix, keys, q->offs + q0, nb, flags, c.ctx, c.obj, c.uctx, c.uobj), "device counting");
    return c;
}

static void free_counts(counts_t *c)
{
    free(c->ctx);
    free(c->obj);
    free(c->uctx);
    free(c->uobj);
}

static kssd_features_t feat_of(const kssdgpu_ctx_mut2_t *c, const kssdgpu_obj_section_t *o)
{
    kssd_features_t f = {0};
    f.XnY_ctx = c->num_ctx;
    f.N_mut2_ctx = c->num_mut2_ctx;
    f.N_diff_obj = o->diff_obj;
    f.N_diff_obj_section = o->diff_obj_section;
    return f;
}

static double naive_of(const kssdgpu_ctx_mut2_t *c, const kssdgpu_obj_section_t *o)
{
    kssd_features_t f = feat_of(c, o);
    return kssd_naive_dist(&f);
}

/* The counters of one (query, reference) cell. */
typedef struct cell {
    kssdgpu_ctx_mut2_t c, uc;
    kssdgpu_obj_section_t o, uo;
} cell_t;

/* Candidates of a detail block from kssdgpu_count_detail: the device applies the
 * pre-filter of src/command_ani.h:585-609 with a margin below anicut, so only these
 * cells (ascending (query, ref)) cross to the host; the host re-applies the exact test. */
typedef struct detail_hits {
    kssdgpu_hit_t *hits;
    uint64_t *row_offs; /* nb + 1 */
} detail_hits_t;

static detail_hits_t detail_candidates(kssdgpu_index_t *ix, const kssd_sketch_t *q, int q0, int nb, unsigned flags,
                                       const uint32_t *qcnt_block, const uint32_t *rcnt, const kssd_ani_opt_t *o)
{
    detail_hits_t d = {0};
    d.row_offs = malloc(((size_t)nb + 1) * sizeof(uint64_t));
    uint64_t cap = (uint64_t)nb * 64;
    d.hits = malloc(cap * sizeof(kssdgpu_hit_t) + 1);
    if (!d.row_offs || !d.hits)
        err(EXIT_FAILURE, "OOM detail candidates");
    const uint64_t *keys = q->keys + (q->offs[q0] - q->offs[0]);
    int rc = kssdgpu_count_detail(ix, keys, q->offs + q0, nb, flags, qcnt_block, rcnt, o->ctxcut, o->afcut, o->anicut,
                                  d.hits, cap, d.row_offs);
    if (rc == KSSDGPU_ERR_CAPACITY) {
        /* more candidates than the first guess: the call reported how many */
        cap = d.row_offs[nb];
        free(d.hits);
        d.hits = malloc(cap * sizeof(kssdgpu_hit_t) + 1);
        if (!d.hits)
            err(EXIT_FAILURE, "OOM detail candidates");
        rc = kssdgpu_count_detail(ix, keys, q->offs + q0, nb, flags, qcnt_block, rcnt, o->ctxcut, o->afcut,
                                  o->anicut, d.hits, cap, d.row_offs);
    }
    gpu_check(rc, "device counting (detail candidates)");
    return d;
}

static cell_t cell_of_hit(const kssdgpu_hit_t *h)
{
    cell_t x;
    x.c.num_ctx = h->num_ctx;
    x.c.num_mut2_ctx = h->num_mut2_ctx;
    x.o.diff_obj = h->diff_obj;
    x.o.diff_obj_section = h->diff_obj_section;
    x.uc.num_ctx = h->u_num_ctx;
    x.uc.num_mut2_ctx = h->u_num_mut2_ctx;
    x.uo.diff_obj = h->u_diff_obj;
    x.uo.diff_obj_section = h->u_diff_obj_section;
    return x;
}

/* query blocks sized so that four counter blocks stay within ~2 GB of host memory */
static int block_for(int nref, int nq)
{
    size_t per = (size_t)nref * 32;
    size_t b = per ? (2ull << 30) / per : (size_t)nq;
    if (b < 1)
        b = 1;
    if (b > 8192)
        b = 8192;
    return (int)(b < (size_t)nq ? b : (size_t)(nq ? nq : 1));
}

/* ------------------------------------------------------------------ ranking (detail pre-filter) */

typedef struct {
    uint32_t id;
    float ani;
} idani_t;

static int cmp_idani_desc(const void *a, const void *b)
{
    const idani_t *x = a, *y = b;
    return (x->ani < y->ani) - (x->ani > y->ani);
}

/* The reference keeps the top N by a partial min-heap before a final sort when N is
 * well below the candidate count (src/command_ani.h:368-433); ties between equal
 * ANIs are resolved by that exact sequence of swaps and sorts, so it is kept. */
static void heap_sift_down(idani_t *h, int n, int i)
{
    for (;;) {
        int l = 2 * i + 1, r = l + 1, s = i;
        if (l < n && h[l].ani < h[s].ani) s = l;
        if (r < n && h[r].ani < h[s].ani) s = r;
        if (s == i) break;
        idani_t t = h[i];
        h[i] = h[s];
        h[s] = t;
        i = s;
    }
}

static int select_topn(idani_t *a, int m, int topn)
{
    if (m <= 0 || topn <= 0)
        return 0;
    if (topn > m)
        topn = m;
    if (m <= 128 || topn >= m / 2) {
        qsort(a, (size_t)m, sizeof *a, cmp_idani_desc);
        return topn;
    }
    for (int i = (topn >> 1) - 1; i >= 0; --i)
        heap_sift_down(a, topn, i);
    for (int i = topn; i < m; ++i) {
        if (a[i].ani <= a[0].ani)
            continue;
        idani_t t = a[i];
        a[i] = a[0];
        a[0] = t;
        heap_sift_down(a, topn, 0);
    }
    qsort(a, (size_t)topn, sizeof *a, cmp_idani_desc);
    return topn;
}

typedef struct {
    double ani;
    uint32_t id;
} urank_t;

static int cmp_urank(const void *a, const void *b)
{
    const urank_t *x = a, *y = b;
    if (x->ani != y->ani)
        return x->ani < y->ani ? 1 : -1;
    return (x->id > y->id) - (x->id < y->id);
}

/* ------------------------------------------------------------------ mem_eff index path */

static void print_unique_block(kssd_buf_t *b, int R, int q0, int nb, const uint32_t *rcnt, const uint32_t *qcnt,
                               const uint32_t *uref, const counts_t *c, char (*refn)[PATHLEN], char (*qryn)[PATHLEN])
{
    /* print_unique_context_block, src/command_ani.c:462-492 */
    for (int q = 0; q < nb; ++q)
        for (int r = 0; r < R; ++r) {
            const size_t cell = (size_t)q * R + r;
            if (!c->ctx[cell].num_ctx)
                continue;
            const uint32_t shared = c->uctx[cell].num_ctx;
            kssd_buf_printf(b, "%s\t%s\t%u\t%u\t%u\t%u\t%u\t%u\t%u\t%u\t%u\t%u\t%u", qryn[q0 + q], refn[r], qcnt[q0 + q],
                            rcnt[r], c->ctx[cell].num_ctx, c->obj[cell].diff_obj, c->obj[cell].diff_obj_section,
                            c->ctx[cell].num_mut2_ctx, uref[r], shared, c->uobj[cell].diff_obj,
                            c->uobj[cell].diff_obj_section, c->uctx[cell].num_mut2_ctx);
            if (shared) {
                kssd_features_t f = feat_of(&c->uctx[cell], &c->uobj[cell]);
                kssd_buf_printf(b, "\t%.6f", 1.0 - kssd_naive_dist(&f));
            } else
                kssd_buf_puts(b, "\tNA");
            kssd_buf_printf(b, "\t%.6f", (double)shared / qcnt[q0 + q]);
            if (uref[r])
                kssd_buf_printf(b, "\t%.6f", (double)shared / uref[r]);
            else
                kssd_buf_puts(b, "\tNA");
            kssd_buf_printf(b, "\t%.6f\n", (double)shared / rcnt[r]);
        }
}

static FILE *open_out_with_report(const char *path, FILE *report)
{
    if (!report)
        return path[0] ? fopen(path, "w") : stdout;
    int fd = path[0] ? open(path, O_WRONLY | O_CREAT, 0666) : STDOUT_FILENO;
    if (fd < 0)
        err(errno, "%s", path);
    struct stat out, diag;
    if (fstat(fd, &out) || fstat(fileno(report), &diag))
        err(errno, "Cannot check ANI output identity");
    if (out.st_dev == diag.st_dev && out.st_ino == diag.st_ino)
        errx(EXIT_FAILURE, "--unique-ctx-report must differ from the ordinary output path");
    if (!path[0])
        return stdout;
    if (S_ISREG(out.st_mode) && ftruncate(fd, 0))
        err(errno, "%s", path);
    FILE *fp = fdopen(fd, "w");
    if (!fp) {
        close(fd);
        err(errno, "%s", path);
    }
    return fp;
}

/* ---- --estimate-coverage inputs */

/* load_coverage_unique_bits (src/command_ani.c:2209-2253): the reference database's
 * marker bits when its index and .unique_bits are both present and sized right */
typedef struct cov_db {
    kssd_cov_refdb_t db;
    uint8_t *bits;
    kssd_index_rec_t *rec;
    bool own_rec;
} cov_db_t;

static void cov_db_load(cov_db_t *c, const char *refdir, uint64_t entries, kssd_index_rec_t *rec)
{
    memset(c, 0, sizeof *c);
    if (!kssd_file_exists(refdir, "sortedcomb_ctxgid64obj32.unique_bits"))
        return;
    if (!kssd_file_exists(refdir, "sortedcomb_ctxgid64obj32")) {
        warnx("load_coverage_unique_bits(): ignoring %s/%s because %s is missing", refdir,
              "sortedcomb_ctxgid64obj32.unique_bits", "sortedcomb_ctxgid64obj32");
        return;
    }
    size_t nbits = 0;
    c->bits = kssd_unique_bits_load(refdir, &nbits);
    if (!c->bits || nbits != (size_t)((entries + 7u) >> 3)) {
        warnx("load_coverage_unique_bits(): ignoring %s/%s: %zu bytes, expected %zu", refdir,
              "sortedcomb_ctxgid64obj32.unique_bits", nbits, (size_t)((entries + 7u) >> 3));
        free(c->bits);
        c->bits = NULL;
        return;
    }
    if (rec) {
        c->rec = rec;
    } else {
        size_t n = 0;
        c->rec = kssd_index_load(refdir, &n);
        c->own_rec = true;
        if (!c->rec || n != entries) {
            warnx("load_coverage_unique_bits(): ignoring %s/%s: %zu records, expected %llu", refdir,
                  "sortedcomb_ctxgid64obj32", n, (unsigned long long)entries);
            free(c->rec);
            free(c->bits);
            memset(c, 0, sizeof *c);
            return;
        }
    }
    c->db.available = true;
    c->db.entries = entries;
    c->db.bits = c->bits;
    c->db.sorted = c->rec;
}

static void cov_db_free(cov_db_t *c)
{
    free(c->bits);
    if (c->own_rec)
        free(c->rec);
    memset(c, 0, sizeof *c);
}

/* the query's per-key counts: mem_eff reads comblco.a when present and sized right
 * (src/command_ani.c:536-551); the streaming paths with the sketch when it was made
 * with counting (SKETCH_PARSE_ABUNDANCE, src/global_basic.c:1123-1124) */
static uint32_t *cov_query_counts(const kssd_sketch_t *q, const char *dir, bool required)
{
    const size_t entries = (size_t)(q->offs[q->n] - q->offs[0]);
    if (!kssd_file_exists(dir, "comblco.a")) {
        if (required)
            errx(EXIT_FAILURE, "%s/comblco.a: missing abundances of a counted sketch", dir);
        return NULL;
    }
    size_t n = 0;
    uint32_t *a = kssd_abundance_load(dir, &n);
    if (!a)
        errx(EXIT_FAILURE, "%s", kssd_host_last_error());
    if (n != entries) {
        if (required)
            errx(EXIT_FAILURE, "%s/comblco.a has %zu counts, expected %zu", dir, n, entries);
        warnx("ani_mem_eff(): ignoring %s/comblco.a: %zu bytes, expected %zu", dir, n * 4, entries * 4);
        free(a);
        return NULL;
    }
    return a;
}

static int run_mem_eff(void)
{
    kssd_ani_opt_t *o = &g.o;
    const bool count_unique = g.unique_ctx || g.unique_report[0];
    kssd_sketch_t *ref = load_sketch(g.refdir, ref_flags());
    kssd_sketch_t *qry = load_sketch(g.qrydir, qry_flags());
    size_t nrec = 0;
    kssd_index_rec_t *rec = kssd_index_load(g.refdir, &nrec);
    if (!rec)
        errx(EXIT_FAILURE, "%s", kssd_host_last_error());
    if (nrec != (size_t)(ref->offs[ref->n] - ref->offs[0]))
        errx(EXIT_FAILURE, "%s/sortedcomb_ctxgid64obj32: %zu records, expected %llu", g.refdir, nrec,
             (unsigned long long)(ref->offs[ref->n] - ref->offs[0]));
    if (qry->stat.hash_id != ref->stat.hash_id)
        errx(EXIT_FAILURE, "hash_id mismatch between query and reference sketches");
    const int R = ref->n;
    kssdgpu_index_t *ix = NULL;
    gpu_check(kssdgpu_index_from_records(rec, nrec, R, qry->obj_bits, 0, &ix), "device index");
    const bool coverage = o->estimate_coverage && o->fmt == 0;
    cov_db_t cov = {0};
    uint32_t *qab = NULL;
    if (coverage) {
        cov_db_load(&cov, g.refdir, nrec, rec);
        qab = cov_query_counts(qry, g.qrydir, false);
    }
    if (!cov.rec)
        free(rec);
    uint32_t *rcnt = malloc((size_t)R * 4 + 4), *uref = malloc((size_t)R * 4 + 4);
    if (ref->stat.conflict)
        gpu_check(kssdgpu_index_ref_ctx_counts(ix, 1, o->ignoreconflict, rcnt, uref), "reference counts");
    else {
        for (int i = 0; i < R; ++i)
            rcnt[i] = (uint32_t)(ref->offs[i + 1] - ref->offs[i]);
        gpu_check(kssdgpu_index_ref_ctx_counts(ix, 0, o->ignoreconflict, NULL, uref), "reference counts");
    }
    uint32_t *qcnt = sample_ctx_counts(qry, qry->stat.conflict, false);

    FILE *report = NULL;
    if (g.unique_report[0]) {
        report = fopen(g.unique_report, "wx");
        if (!report)
            err(errno, "%s", g.unique_report);
        fprintf(report, "Qry\tRef\tQry_ctx\tRef_ctx\tXnY_ctx\tN_diff_obj\tN_diff_obj_section\tN_mut2_ctx\tUnique_Ref_ctx\t"
                        "Unique_XnY_ctx\tUnique_N_diff_obj\tUnique_N_diff_obj_section\tUnique_N_mut2_ctx\tUnique_ANI\t"
                        "Unique_QAF\tUnique_RAF\tUnique_RAF_fullref\n");
    }
    FILE *out = open_out_with_report(g.outf, report);
    if (!out)
        err(errno, "%s", g.outf);
    kssd_buf_t hb = {0};
    if (o->fmt) {
        for (int i = 0; i < R; ++i) {
            kssd_buf_putc(&hb, '\t');
            kssd_buf_puts(&hb, ref->names[i]);
        }
        kssd_buf_putc(&hb, '\n');
    } else {
        kssd_buf_puts(&hb, kssd_detail_header);
        if (coverage) {
            kssd_buf_putc(&hb, '\t');
            kssd_buf_puts(&hb, kssd_coverage_header);
        }
        kssd_buf_putc(&hb, '\n');
    }
    write_buf(out, &hb);
    kssd_buf_free(&hb);

    const unsigned flags = (o->ignoreconflict ? KSSDGPU_IGNORECONFLICT : 0) | (count_unique ? KSSDGPU_UNIQUE : 0);
    const int ntop = o->ntop > 0 ? o->ntop : R;
    const int B = block_for(R, qry->n);
    /* detail mode keeps the dense counters on the device and takes only its candidates;
     * the unique-context report prints every cell, so it takes the dense block */
    const bool sparse = !o->fmt && !report;
    for (int q0 = 0; q0 < qry->n; q0 += B) {
        const int nb = qry->n - q0 < B ? qry->n - q0 : B;
        counts_t c = {0};
        detail_hits_t dh = {0};
        if (sparse)
            dh = detail_candidates(ix, qry, q0, nb, flags, qcnt + q0, rcnt, o);
        else
            c = count_queries(ix, R, qry, q0, nb, flags);
        if (report) {
            kssd_buf_t rb = {0};
            print_unique_block(&rb, R, q0, nb, rcnt, qcnt, uref, &c, ref->names, qry->names);
            write_buf(report, &rb);
            kssd_buf_free(&rb);
        }
        kssd_buf_t *rows = calloc((size_t)nb, sizeof(kssd_buf_t));
#pragma omp parallel for schedule(dynamic, 1) num_threads(o->p)
        for (int i = 0; i < nb; ++i) {
            const int qg = q0 + i;
            const size_t a_size = (size_t)(qry->offs[qg + 1] - qry->offs[qg]);
            kssd_buf_t *b = &rows[i];
            const kssdgpu_ctx_mut2_t *cx = c.ctx ? c.ctx + (size_t)i * R : NULL;
            const kssdgpu_obj_section_t *ob = c.obj ? c.obj + (size_t)i * R : NULL;
            const kssdgpu_ctx_mut2_t *ucx = c.uctx ? c.uctx + (size_t)i * R : NULL;
            const kssdgpu_obj_section_t *uob = c.uobj ? c.uobj + (size_t)i * R : NULL;
            /* this query's cells: the dense row, or its device candidates (ascending ref) */
            const kssdgpu_hit_t *hq = sparse ? dh.hits + dh.row_offs[i] : NULL;
            const int hn = sparse ? (int)(dh.row_offs[i + 1] - dh.row_offs[i]) : 0;
            cell_t *cells = sparse ? malloc((size_t)(hn ? hn : 1) * sizeof(cell_t)) : NULL;
            for (int k = 0; k < hn; ++k)
                cells[k] = cell_of_hit(&hq[k]);
            uint32_t *ids = NULL;
            int out_n = 0;
            if (!o->fmt) {
                /* detail candidates and ranking, src/command_ani.h:577-621 */
                if (a_size) {
                    const int span = sparse ? hn : R;
                    idani_t *cand = malloc((size_t)span * sizeof(idani_t) + 8);
                    urank_t *ranks = o->unique_ctx ? malloc((size_t)span * sizeof(urank_t) + 16) : NULL;
                    int m = 0;
                    for (int k = 0; k < span; ++k) {
                        const int j = sparse ? (int)hq[k].ref : k;
                        const kssdgpu_ctx_mut2_t *cj = sparse ? &cells[k].c : &cx[j];
                        const kssdgpu_obj_section_t *oj = sparse ? &cells[k].o : &ob[j];
                        const uint32_t shared = cj->num_ctx;
                        if (shared < (uint32_t)o->ctxcut)
                            continue;
                        if (rcnt[j] == 0 || qcnt[qg] == 0 ||
                            !kssd_af_pass(o, (double)shared / (double)qcnt[qg], (double)shared / (double)rcnt[j]))
                            continue;
                        float dist = (float)oj->diff_obj / cj->num_ctx / 7;
                        double ani = (float)(1 - dist);
                        if (ranks) {
                            const kssdgpu_ctx_mut2_t *ucj = sparse ? &cells[k].uc : &ucx[j];
                            const kssdgpu_obj_section_t *uoj = sparse ? &cells[k].uo : &uob[j];
                            const bool use_u = kssd_use_unique_context(ucj->num_ctx, rcnt[j]);
                            ani = 1.0 - (use_u ? naive_of(ucj, uoj) : naive_of(cj, oj));
                        }
                        if (ani < o->anicut)
                            continue;
                        if (ranks)
                            ranks[m] = (urank_t){ani, (uint32_t)j};
                        cand[m].id = (uint32_t)j;
                        cand[m].ani = (float)ani;
                        m++;
                    }
                    ids = malloc((size_t)(m ? m : 1) * sizeof(uint32_t));
                    if (ranks) {
                        qsort(ranks, (size_t)m, sizeof *ranks, cmp_urank);
                        out_n = m < ntop ? m : ntop;
                        for (int r = 0; r < out_n; ++r)
                            ids[r] = ranks[r].id;
                        free(ranks);
                    } else {
                        out_n = select_topn(cand, m, ntop);
                        for (int r = 0; r < out_n; ++r)
                            ids[r] = cand[r].id;
                    }
                    free(cand);
                }
            } else {
                kssd_buf_puts(b, qry->names[qg]);
            }
            const int loop = o->fmt ? R : out_n;
            const int qsize = (int)qcnt[qg];
            /* with coverage the reported rows are collected, their coverage computed
             * together, then printed (ani_block_print_internal, src/command_ani.c:3452-3544) */
            kssd_row_t *cov_rows = coverage ? malloc((size_t)(loop ? loop : 1) * sizeof(kssd_row_t)) : NULL;
            size_t cov_n = 0;
            for (int n = 0; n < loop; ++n) {
                const int j = o->fmt ? n : (int)ids[n];
                cell_t cl = {0};
                if (sparse) {
                    /* the candidate of reference j (candidates ascend by ref) */
                    int lo = 0, hi = hn - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if ((int)hq[mid].ref < j)
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    cl = cells[lo];
                } else {
                    cl.c = cx[j];
                    cl.o = ob[j];
                    if (ucx) {
                        cl.uc = ucx[j];
                        cl.uo = uob[j];
                    }
                }
                kssd_features_t f = feat_of(&cl.c, &cl.o);
                const int rsize = (int)rcnt[j];
                if (qsize == 0 || rsize == 0) {
                    if (o->fmt)
                        kssd_buf_printf(b, "\t%lf", kssd_matrix_exception_value(o));
                    continue;
                }
                /* this path reports single-precision align fractions (src/command_ani.c:3489-3494) */
                const float af_q = (float)f.XnY_ctx / qsize;
                const float af_r = (float)f.XnY_ctx / rsize;
                f.X_ctx = (uint32_t)qsize;
                const float bq = (float)kssd_af_anib(&f, o->drfold);
                f.X_ctx = (uint32_t)rsize;
                const float br = (float)kssd_af_anib(&f, o->drfold);
                kssd_row_t row = kssd_make_row((uint32_t)j, &f, o, (uint32_t)qsize, (uint32_t)rsize, af_q, bq, af_r, br,
                                               qry->meta ? &qry->meta[qg] : NULL, ref->meta ? &ref->meta[j] : NULL);
                if (o->unique_ctx) {
                    row.unique_ctx_selected = kssd_use_unique_context(cl.uc.num_ctx, rcnt[j]);
                    row.naive_dist = row.unique_ctx_selected ? naive_of(&cl.uc, &cl.uo) : naive_of(&cl.c, &cl.o);
                    kssd_finalize_row(&row, o);
                }
                const double metric = o->s < 0 ? row.selected_ani : row.metric;
                if (o->fmt)
                    kssd_buf_printf(b, "\t%lf", metric);
                else if (row.selected_ani >= o->anicut) {
                    if (coverage)
                        cov_rows[cov_n++] = row;
                    else
                        kssd_append_detail_row(b, o, qry->names[qg], ref->names[j], &row, anno_at(ref, (uint32_t)j));
                }
            }
            if (coverage && cov_n) {
                const size_t qb = (size_t)(qry->offs[qg] - qry->offs[0]);
                kssd_coverage_rows(qry->keys + qb, qab ? qab + qb : NULL, a_size, ref->keys, ref->offs,
                                   cov.db.available ? &cov.db : NULL, qry->obj_bits, cov_rows, cov_n);
                for (size_t k = 0; k < cov_n; ++k)
                    kssd_append_detail_row(b, o, qry->names[qg], ref->names[cov_rows[k].rn], &cov_rows[k],
                                           anno_at(ref, cov_rows[k].rn));
            }
            free(cov_rows);
            if (o->fmt)
                kssd_buf_putc(b, '\n');
            free(ids);
            free(cells);
        }
        for (int i = 0; i < nb; ++i) {
            write_buf(out, &rows[i]);
            kssd_buf_free(&rows[i]);
        }
        free(rows);
        free_counts(&c);
        free(dh.hits);
        free(dh.row_offs);
    }
    if (report && fclose(report) != 0)
        err(errno, "Cannot finish unique-context report");
    close_out(out);
    kssdgpu_index_free(ix);
    free(rcnt);
    free(uref);
    free(qcnt);
    free(qab);
    free(cov.rec);
    cov_db_free(&cov);
    kssd_sketch_free(ref);
    kssd_sketch_free(qry);
    return 0;
}

/* ------------------------------------------------------------------ self matrices */

/* Writes sortedcomb_ctxgid64obj32 and its unique bits from the device index, as
 * `kssd3a sketch -i` does (gen_inverted_index4comblco, src/command_sketch.c:916-938). */
static void write_index_files(const char *dir, kssdgpu_index_t *ix, uint64_t n)
{
    kssd_index_rec_t *rec = malloc(n * sizeof(*rec) + 12);
    uint8_t *bits = malloc((n + 7) / 8 + 1);
    if (!rec || !bits)
        err(EXIT_FAILURE, "OOM index export");
    gpu_check(kssdgpu_index_export(ix, rec, bits), "index export");
    if (kssd_index_write(dir, rec, n, bits))
        errx(EXIT_FAILURE, "%s", kssd_host_last_error());
    uint64_t marked = 0;
    for (uint64_t i = 0; i < n; ++i)
        marked += (bits[i >> 3] >> (i & 7)) & 1u;
    fprintf(stderr, "sketch unique-index: wrote %s/sortedcomb_ctxgid64obj32.unique_bits (%llu bytes; %llu unique markers / %llu records)\n",
            dir, (unsigned long long)((n + 7) / 8), (unsigned long long)marked, (unsigned long long)n);
    free(rec);
    free(bits);
}

/* Order-independent checksum of (ctxgid, obj) over index records or over a sketch's
 * entries: equal sums (with equal counts) show the index file was built from this
 * sketch, so the self join over it gives count_lower's counters. */
static uint64_t mix_rec(uint64_t ctxgid, uint32_t obj)
{
    uint64_t x = ctxgid * 0x9E3779B97F4A7C15ull ^ ((uint64_t)obj + 0x632BE59BD9B4E019ull);
    x ^= x >> 31;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 29;
    return x;
}

static uint64_t records_checksum(const kssd_index_rec_t *rec, size_t n)
{
    uint64_t sum = 0;
#pragma omp parallel for reduction(+ : sum) schedule(static) num_threads(g.o.p)
    for (size_t i = 0; i < n; ++i)
        sum += mix_rec(rec[i].ctxgid, rec[i].obj);
    return sum;
}

static uint64_t sketch_checksum(const kssd_sketch_t *s)
{
    uint64_t sum = 0;
    const uint64_t objmask = s->obj_bits >= 64 ? ~0ull : ((1ull << s->obj_bits) - 1);
#pragma omp parallel for reduction(+ : sum) schedule(dynamic, 16) num_threads(g.o.p)
    for (int gid = 0; gid < s->n; ++gid)
        for (uint64_t i = s->offs[gid]; i < s->offs[gid + 1]; ++i) {
            const uint64_t k = s->keys[i - s->offs[0]];
            sum += mix_rec(((k >> s->obj_bits) << KSSD_GID_BITS) | (uint64_t)gid, (uint32_t)(k & objmask));
        }
    return sum;
}

/* Lower-triangle counters of a self sketch.  With an index file the reference reads
 * that index: when its records are the sketch's own (checksum), the self join over it
 * gives the same counters; otherwise the probe kernel runs the sketch's queries
 * against it.  Without a file, the self join over the index the device builds. */
static void self_lower_counts(const kssd_sketch_t *s, const char *dir, bool index_file, bool forced_needs_file,
                              kssdgpu_ctx_mut2_t **pc, kssdgpu_obj_section_t **po)
{
    const int n = s->n;
    const size_t cells = (size_t)n * (n - 1) / 2;
    kssdgpu_ctx_mut2_t *lc = malloc(cells * sizeof(*lc) + 8);
    kssdgpu_obj_section_t *lo = malloc(cells * sizeof(*lo) + 8);
    if (!lc || !lo)
        err(EXIT_FAILURE, "OOM lower triangle");
    /* map the pages on all cores before the device copies land there: a copy into
     * untouched memory runs at page-fault speed */
    const size_t pieces = (cells * sizeof(*lc) + (8u << 20) - 1) / (8u << 20);
#pragma omp parallel for schedule(dynamic, 1) num_threads(g.o.p)
    for (size_t k = 0; k < pieces; ++k) {
        const size_t off = k * (8u << 20), len = cells * sizeof(*lc) - off < (8u << 20) ? cells * sizeof(*lc) - off
                                                                                         : (8u << 20);
        memset((char *)lc + off, 0, len);
        memset((char *)lo + off, 0, len);
    }
    const unsigned flags = g.o.ignoreconflict ? KSSDGPU_IGNORECONFLICT : 0;
    if (index_file) {
        size_t nrec = 0;
        kssd_index_rec_t *rec = kssd_index_load(dir, &nrec);
        if (!rec)
            errx(EXIT_FAILURE, "%s", kssd_host_last_error());
        if (nrec != (size_t)(s->offs[n] - s->offs[0]))
            errx(EINVAL, "load_self_sorted_index_or_build(): sorted index size mismatch");
        phase("read index file");
        const bool own = records_checksum(rec, nrec) == sketch_checksum(s);
        phase("index/sketch checksum");
        kssdgpu_index_t *ix = NULL;
        gpu_check(kssdgpu_index_from_records(rec, nrec, n, s->obj_bits, 0, &ix), "device index");
        free(rec);
        phase("device index from records");
        if (own) {
            if (cells)
                gpu_check(kssdgpu_self_lower(ix, flags, lc, lo), "device self join");
            phase("self join + D2H");
        } else {
            const int B = block_for(n, n);
            for (int q0 = 0; q0 < n; q0 += B) {
                const int nb = n - q0 < B ? n - q0 : B;
                kssdgpu_ctx_mut2_t *c = malloc((size_t)nb * n * sizeof(*c) + 8);
                kssdgpu_obj_section_t *o = malloc((size_t)nb * n * sizeof(*o) + 8);
                if (!c || !o)
                    err(EXIT_FAILURE, "OOM counter block");
                gpu_check(kssdgpu_count_lower(ix, s->keys + (s->offs[q0] - s->offs[0]), s->offs + q0, nb, q0, flags, c,
                                              o),
                          "device counting");
#pragma omp parallel for schedule(static) num_threads(g.o.p)
                for (int i = 0; i < nb; ++i) {
                    const int q = q0 + i;
                    if (q == 0)
                        continue;
                    memcpy(lc + (size_t)q * (q - 1) / 2, c + (size_t)i * n, (size_t)q * sizeof(*c));
                    memcpy(lo + (size_t)q * (q - 1) / 2, o + (size_t)i * n, (size_t)q * sizeof(*o));
                }
                free(c);
                free(o);
            }
            phase("probe count_lower + D2H");
        }
        kssdgpu_index_free(ix);
    } else {
        if (forced_needs_file && force_ref_index())
            errx(EXIT_FAILURE, "KSSD3A_FORCE_REF_INDEX requires reference index '%s/%s'", dir,
                 "sortedcomb_ctxgid64obj32");
        kssdgpu_index_t *ix = gpu_index_of_sketch(s);
        phase("device index from sketch");
        if (cells)
            gpu_check(kssdgpu_self_lower(ix, flags, lc, lo), "device self join");
        phase("self join + D2H");
        kssdgpu_index_free(ix);
    }
    *pc = lc;
    *po = lo;
}

/* One self-matrix cell valued on the host (the zero-overlap constant, or the pair metric). */
static double self_cell_metric(const kssd_sketch_t *s, const uint32_t *qcnt, const uint32_t *rcnt, int q, int r,
                               const kssdgpu_ctx_mut2_t *c, const kssdgpu_obj_section_t *o, bool zero_const,
                               double zero_metric)
{
    if (zero_const && c->num_ctx == 0 && qcnt[q] && rcnt[r])
        return zero_metric;
    kssd_features_t f = feat_of(c, o);
    return kssd_pair_metric(&f, qcnt[q], rcnt[r], &g.o, s->meta ? &s->meta[q] : NULL, s->meta ? &s->meta[r] : NULL);
}

/* metric values of every lower pair (q > r), rows in parallel */
static double *self_lower_metrics(const kssd_sketch_t *s, const kssdgpu_ctx_mut2_t *lc, const kssdgpu_obj_section_t *lo)
{
    const int n = s->n;
    const size_t cells = (size_t)n * (n - 1) / 2;
    uint32_t *qcnt = sample_ctx_counts(s, s->stat.conflict, false);
    uint32_t *rcnt = g.o.ignoreconflict ? sample_ctx_counts(s, s->stat.conflict, true) : qcnt;
    double *m = malloc(cells * sizeof(double) + 8);
    if (!m)
        err(EXIT_FAILURE, "OOM metrics");
    double zero_metric = 0;
    const bool zero_const = kssd_zero_overlap_metric(&g.o, &zero_metric);
#pragma omp parallel for schedule(dynamic, 16) num_threads(g.o.p)
    for (int q = 1; q < n; ++q) {
        const size_t base = (size_t)q * (q - 1) / 2;
        for (int r = 0; r < q; ++r)
            m[base + r] = self_cell_metric(s, qcnt, rcnt, q, r, &lc[base + r], &lo[base + r], zero_const, zero_metric);
    }
    phase("epilogue (host FP64)");
    if (rcnt != qcnt)
        free(rcnt);
    free(qcnt);
    return m;
}

static void print_self_full_fixed6(const kssd_sketch_t *s, const double *m)
{
    /* comb_sortedsketch64_indexed_self_full printing, src/command_ani.c:1711-1746.
     * Rows go out in chunks of B: the chunk's scaled values are first gathered into a
     * B x n tile (the lower triangle read along rows for r < q and along columns for
     * r > q, both contiguous), then rows are formatted in parallel from the tile while
     * the previous chunk is being written. */
    const int n = s->n;
    FILE *out = open_out(g.outf);
    kssd_buf_t h = {0};
    for (int r = 0; r < n; ++r) {
        kssd_buf_putc(&h, '\t');
        kssd_buf_puts(&h, s->names[r]);
    }
    kssd_buf_putc(&h, '\n');
    write_buf(out, &h);
    kssd_buf_free(&h);
    const int32_t diag = kssd_scale_fixed6(kssd_matrix_diagonal_value(&g.o));
    const int B = 256;
    int32_t *tile = malloc((size_t)B * (size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    if (!tile)
        err(EXIT_FAILURE, "OOM output tile");
    const int threads = g.o.p > 0 ? g.o.p : 1;
    int cb = n / (threads * 4);
    if (cb < 64)
        cb = 64;
    owriter_t w;
    owriter_start(&w, out);
    for (int q0 = 0; q0 < n; q0 += B) {
        const int nb = n - q0 < B ? n - q0 : B;
#pragma omp parallel for schedule(dynamic, 1) num_threads(g.o.p)
        for (int rb = 0; rb < n; rb += cb) {
            const int re = n - rb < cb ? n : rb + cb;
            for (int i = 0; i < nb; ++i) {
                /* r < q: row q of the triangle */
                const int q = q0 + i;
                int32_t *t = tile + (size_t)i * n;
                const double *mq = m + (size_t)q * (size_t)(q > 0 ? q - 1 : 0) / 2;
                const int e = re < q ? re : q;
                for (int r = rb; r < e; ++r)
                    t[r] = kssd_scale_fixed6(mq[r]);
                if (q >= rb && q < re)
                    t[q] = diag;
            }
            for (int r = rb; r < re; ++r) {
                /* r > q: column q of the triangle, contiguous over the chunk's rows */
                const int iend = r - q0 < nb ? r - q0 : nb;
                if (iend <= 0)
                    continue;
                const double *mr = m + (size_t)r * (size_t)(r - 1) / 2 + q0;
                for (int i = 0; i < iend; ++i)
                    tile[(size_t)i * n + r] = kssd_scale_fixed6(mr[i]);
            }
        }
        kssd_buf_t *rows = calloc((size_t)nb, sizeof(kssd_buf_t));
        if (!rows)
            err(EXIT_FAILURE, "OOM output rows");
#pragma omp parallel for schedule(dynamic, 1) num_threads(g.o.p)
        for (int i = 0; i < nb; ++i) {
            kssd_buf_t *b = &rows[i];
            const int32_t *t = tile + (size_t)i * n;
            kssd_buf_reserve(b, (size_t)n * 10 + PATHLEN);
            kssd_buf_puts(b, s->names[q0 + i]);
            for (int r = 0; r < n; ++r) {
                kssd_buf_putc(b, '\t');
                kssd_put_scaled6(b, t[r]);
            }
            kssd_buf_putc(b, '\n');
        }
        owriter_push(&w, rows, nb);
    }
    owriter_finish(&w);
    free(tile);
    close_out(out);
}

static void print_self_lf(const kssd_sketch_t *s, const double *m, bool full)
{
    /* "%lf" matrices: direct full (src/command_ani.c:3320-3343) and triangles (:1809-1822,:3346-3357) */
    const int n = s->n;
    FILE *out = open_out(g.outf);
    if (full) {
        kssd_buf_t h = {0};
        for (int r = 0; r < n; ++r) {
            kssd_buf_putc(&h, '\t');
            kssd_buf_puts(&h, s->names[r]);
        }
        kssd_buf_putc(&h, '\n');
        write_buf(out, &h);
        kssd_buf_free(&h);
    }
    const double diag = kssd_matrix_diagonal_value(&g.o);
    const int chunk = 256;
    for (int q0 = 0; q0 < n; q0 += chunk) {
        const int nb = n - q0 < chunk ? n - q0 : chunk;
        kssd_buf_t *rows = calloc((size_t)nb, sizeof(kssd_buf_t));
#pragma omp parallel for schedule(dynamic, 1) num_threads(g.o.p)
        for (int i = 0; i < nb; ++i) {
            const int q = q0 + i;
            kssd_buf_t *b = &rows[i];
            kssd_buf_puts(b, s->names[q]);
            const int end = full ? n : q;
            for (int r = 0; r < end; ++r) {
                double v = diag;
                if (q > r)
                    v = m[(size_t)q * (q - 1) / 2 + r];
                else if (q < r)
                    v = m[(size_t)r * (r - 1) / 2 + q];
                kssd_buf_printf(b, "\t%lf", v);
            }
            if (!full && g.o.d)
                kssd_buf_printf(b, "\t%lf", diag);
            kssd_buf_putc(b, '\n');
        }
        for (int i = 0; i < nb; ++i) {
            write_buf(out, &rows[i]);
            kssd_buf_free(&rows[i]);
        }
        free(rows);
    }
    close_out(out);
}

/* The self matrix's values with the FP64 epilogue on the device (kssdgpu_self_lower_metric):
 * 8 bytes per cell come back instead of 16 bytes of counters, and the few cells whose
 * printed digits depend on how a libm rounds log / log1p / pow are recomputed here with
 * the host's.  NULL when the device's list of those cells overflows (the caller then
 * takes the counters path). */
static double *self_values_on_device(const kssd_sketch_t *s, kssdgpu_index_t *ix, unsigned flags)
{
    const int n = s->n;
    const size_t cells = (size_t)n * (n - 1) / 2;
    uint32_t *qcnt = sample_ctx_counts(s, s->stat.conflict, false);
    uint32_t *rcnt = g.o.ignoreconflict ? sample_ctx_counts(s, s->stat.conflict, true) : qcnt;
    double zero_metric = 0;
    const bool zero_const = kssd_zero_overlap_metric(&g.o, &zero_metric);
    kssdgpu_metric_opt_t mo = {0};
    mo.s = g.o.s;
    mo.e = g.o.e;
    mo.v = g.o.v;
    mo.unassembled = g.o.unassembled;
    mo.unified_metric = g.o.unified_metric;
    mo.raw_output = g.o.raw_output;
    mo.afcut = g.o.afcut;
    mo.drfold = g.o.drfold;
    mo.obj_bits = g.o.obj_bits;
    mo.ctx_bits = g.o.ctx_bits;
    mo.zero_const = zero_const;
    mo.zero_value = zero_metric;
    mo.hgb_nodes = kssd_hgb_nodes;
    mo.hgb_nodes_count = KSSD_HGB_NODES;
    mo.hgb_tree_begin = kssd_hgb_tree_begin;
    mo.hgb_trees = KSSD_HGB_TREES;
    mo.hgb_baseline = kssd_hgb_baseline;
    double *m = malloc(cells * sizeof(double) + 8);
    const uint64_t cap = 65536;
    kssdgpu_recheck_t *re = malloc(cap * sizeof(*re));
    if (!m || !re)
        err(EXIT_FAILURE, "OOM matrix values");
    /* map the pages on all cores before the device copy lands there */
    const size_t bytes = cells * sizeof(double), piece = 8u << 20;
    const size_t pieces = (bytes + piece - 1) / piece;
#pragma omp parallel for schedule(dynamic, 1) num_threads(g.o.p)
    for (size_t k = 0; k < pieces; ++k)
        memset((char *)m + k * piece, 0, bytes - k * piece < piece ? bytes - k * piece : piece);
    uint64_t nre = 0;
    const int rc = kssdgpu_self_lower_metric(ix, flags, &mo, qcnt, rcnt, m, re, cap, &nre);
    if (rc == KSSDGPU_ERR_CAPACITY) {
        free(m);
        m = NULL;
    } else {
        gpu_check(rc, "device self join and matrix values");
        for (uint64_t i = 0; i < nre; ++i) {
            const uint64_t cell = re[i].cell;
            int q = (int)((1.0 + sqrt(1.0 + 8.0 * (double)cell)) / 2.0);
            while ((uint64_t)q * (q - 1) / 2 > cell)
                --q;
            while ((uint64_t)(q + 1) * q / 2 <= cell)
                ++q;
            const int r = (int)(cell - (uint64_t)q * (q - 1) / 2);
            m[cell] = self_cell_metric(s, qcnt, rcnt, q, r, &re[i].ctx, &re[i].obj, zero_const, zero_metric);
        }
    }
    free(re);
    if (rcnt != qcnt)
        free(rcnt);
    free(qcnt);
    return m;
}

/* The self matrix's values: on the device where the index is the sketch's own (built
 * from it, or an index file of the same records), else from counters valued on the host. */
static double *self_lower_values(const kssd_sketch_t *s, const char *dir, bool index_file, bool forced_needs_file)
{
    const int n = s->n;
    const size_t cells = (size_t)n * (n - 1) / 2;
    const unsigned flags = g.o.ignoreconflict ? KSSDGPU_IGNORECONFLICT : 0;
    if (cells && getenv("KSSDGPU_HOST_EPILOGUE") == NULL) {
        kssdgpu_index_t *ix = NULL;
        if (index_file) {
            size_t nrec = 0;
            kssd_index_rec_t *rec = kssd_index_load(dir, &nrec);
            if (!rec)
                errx(EXIT_FAILURE, "%s", kssd_host_last_error());
            if (nrec != (size_t)(s->offs[n] - s->offs[0]))
                errx(EINVAL, "load_self_sorted_index_or_build(): sorted index size mismatch");
            phase("read index file");
            const bool own = records_checksum(rec, nrec) == sketch_checksum(s);
            phase("index/sketch checksum");
            free(rec);
            if (own) {
                /* the file holds the sketch's own index: the device builds the same index from
                 * the sketch's keys (2/3 of the file's bytes to move) */
                ix = gpu_index_of_sketch(s);
                phase("device index from sketch");
            }
        } else {
            if (forced_needs_file && force_ref_index())
                errx(EXIT_FAILURE, "KSSD3A_FORCE_REF_INDEX requires reference index '%s/%s'", dir,
                     "sortedcomb_ctxgid64obj32");
            ix = gpu_index_of_sketch(s);
            phase("device index from sketch");
        }
        if (ix) {
            double *m = self_values_on_device(s, ix, flags);
            kssdgpu_index_free(ix);
            phase("self join + device epilogue + D2H");
            if (m)
                return m;
        }
    }
    kssdgpu_ctx_mut2_t *lc = NULL;
    kssdgpu_obj_section_t *lo = NULL;
    self_lower_counts(s, dir, index_file, forced_needs_file, &lc, &lo);
    double *m = self_lower_metrics(s, lc, lo);
    free(lc);
    free(lo);
    return m;
}

/* kind: 0 indexed full (fixed6), 1 indexed triangle, 2 direct (full or triangle per fmt) */
static int run_self(int kind)
{
    phase("start");
    kssd_sketch_t *s = load_sketch(g.qrydir, 0);
    init_bits(s);
    phase("read sketch");
    bool index_file = false;
    if (kind == 0) {
        /* ensure_sorted_ref_index_for_ani_m1 (src/command_ani_wrapper.c:708-716): write the index when absent */
        if (!kssd_file_exists(g.qrydir, "sortedcomb_ctxgid64obj32")) {
            kssdgpu_index_t *ix = gpu_index_of_sketch(s);
            write_index_files(g.qrydir, ix, s->offs[s->n] - s->offs[0]);
            kssdgpu_index_free(ix);
        }
        index_file = true;
    } else if (kind == 1) {
        index_file = kssd_file_exists(g.qrydir, "sortedcomb_ctxgid64obj32");
    }
    double *m = self_lower_values(s, g.qrydir, index_file, kind != 2);
    if (kind == 0)
        print_self_full_fixed6(s, m);
    else if (kind == 1)
        print_self_lf(s, m, false);
    else
        print_self_lf(s, m, g.o.fmt == 1);
    phase("format + write");
    free(m);
    kssd_sketch_free(s);
    return 0;
}

/* ------------------------------------------------------------------ direct rectangular matrix */

static int run_rect_matrix(void)
{
    kssd_sketch_t *qry = load_sketch(g.qrydir, qry_flags());
    kssd_sketch_t *ref = load_sketch(g.refdir, ref_flags());
    kssd_ani_opt_t *o = &g.o;
    uint32_t *qcnt = sample_ctx_counts(qry, qry->stat.conflict, false);
    uint32_t *rcnt = sample_ctx_counts(ref, ref->stat.conflict, o->ignoreconflict);
    kssdgpu_index_t *ix = gpu_index_of_sketch(ref);
    const unsigned flags = (o->ignoreconflict && ref->stat.conflict) ? KSSDGPU_IGNORECONFLICT : 0;
    FILE *out = open_out(g.outf);
    kssd_buf_t h = {0};
    for (int r = 0; r < ref->n; ++r) {
        kssd_buf_putc(&h, '\t');
        kssd_buf_puts(&h, ref->names[r]);
    }
    kssd_buf_putc(&h, '\n');
    write_buf(out, &h);
    kssd_buf_free(&h);
    const int R = ref->n, B = block_for(R, qry->n);
    for (int q0 = 0; q0 < qry->n; q0 += B) {
        const int nb = qry->n - q0 < B ? qry->n - q0 : B;
        counts_t c = count_queries(ix, R, qry, q0, nb, flags);
        kssd_buf_t *rows = calloc((size_t)nb, sizeof(kssd_buf_t));
        double zero_metric = 0;
        const bool zero_const = kssd_zero_overlap_metric(o, &zero_metric);
#pragma omp parallel for schedule(dynamic, 1) num_threads(o->p)
        for (int i = 0; i < nb; ++i) {
            const int q = q0 + i;
            kssd_buf_puts(&rows[i], qry->names[q]);
            for (int r = 0; r < R; ++r) {
                kssd_features_t f = feat_of(&c.ctx[(size_t)i * R + r], &c.obj[(size_t)i * R + r]);
                const double v = (zero_const && f.XnY_ctx == 0 && qcnt[q] && rcnt[r])
                                     ? zero_metric
                                     : kssd_pair_metric(&f, qcnt[q], rcnt[r], o, qry->meta ? &qry->meta[q] : NULL,
                                                        ref->meta ? &ref->meta[r] : NULL);
                kssd_buf_printf(&rows[i], "\t%lf", v);
            }
            kssd_buf_putc(&rows[i], '\n');
        }
        for (int i = 0; i < nb; ++i) {
            write_buf(out, &rows[i]);
            kssd_buf_free(&rows[i]);
        }
        free(rows);
        free_counts(&c);
    }
    close_out(out);
    kssdgpu_index_free(ix);
    free(qcnt);
    free(rcnt);
    kssd_sketch_free(qry);
    kssd_sketch_free(ref);
    return 0;
}

/* ------------------------------------------------------------------ detail paths without an index */

enum { DETAIL_STREAM_ONE = 0, DETAIL_STREAM_MULTI = 1, DETAIL_HASH = 2 };

static int run_detail_scan(int kind)
{
    kssd_ani_opt_t *o = &g.o;
    kssd_sketch_t *qry = load_sketch(g.qrydir, qry_flags());
    kssd_sketch_t *ref = load_sketch(g.refdir, ref_flags());
    if (ref->stat.hash_id != qry->stat.hash_id)
        errx(EXIT_FAILURE, "hash_id mismatch between query and reference sketches");
    const int R = ref->n;
    const bool ref_conflict = ref->stat.conflict;
    /* per-path context counts */
    uint32_t *qcnt, *rcnt, *rtotal;
    if (kind == DETAIL_HASH) {
        qcnt = sample_ctx_counts(qry, qry->stat.conflict, false);
        rcnt = sample_ctx_counts(ref, ref_conflict, o->ignoreconflict);
        rtotal = rcnt;
    } else {
        qcnt = sample_ctx_counts(qry, true, false);
        rcnt = sample_ctx_counts(ref, true, o->ignoreconflict);
        rtotal = kind == DETAIL_STREAM_ONE ? sample_ctx_counts(ref, ref_conflict, o->ignoreconflict) : rcnt;
    }
    kssdgpu_index_t *ix = gpu_index_of_sketch(ref);
    const unsigned flags = kind == DETAIL_HASH ? ((o->ignoreconflict && ref_conflict) ? KSSDGPU_IGNORECONFLICT : 0)
                                               : (o->ignoreconflict ? KSSDGPU_IGNORECONFLICT : 0);
    /* --estimate-coverage: the streaming paths fill the columns (src/command_ani.c:2519,
     * 2641,2822,2989); the no-index hash path prints them as not computed */
    cov_db_t cov = {0};
    uint32_t *qab = NULL;
    if (o->estimate_coverage) {
        if (qry->stat.koc)
            qab = cov_query_counts(qry, g.qrydir, true);
        if (kind != DETAIL_HASH)
            cov_db_load(&cov, g.refdir, (uint64_t)(ref->offs[R] - ref->offs[0]), NULL);
    }
    FILE *out = open_out(g.outf);
    kssd_buf_t h = {0};
    kssd_buf_puts(&h, kssd_detail_header);
    if (o->estimate_coverage) {
        kssd_buf_putc(&h, '\t');
        kssd_buf_puts(&h, kssd_coverage_header);
    }
    kssd_buf_putc(&h, '\n');
    write_buf(out, &h);
    kssd_buf_free(&h);
    const int B = block_for(R, qry->n);
    for (int q0 = 0; q0 < qry->n; q0 += B) {
        const int nb = qry->n - q0 < B ? qry->n - q0 : B;
        counts_t c = count_queries(ix, R, qry, q0, nb, flags);
        kssd_buf_t *rows = calloc((size_t)nb, sizeof(kssd_buf_t));
#pragma omp parallel for schedule(dynamic, 1) num_threads(o->p)
        for (int i = 0; i < nb; ++i) {
            const int q = q0 + i;
            kssd_row_t *surv = malloc((size_t)(R ? R : 1) * sizeof(kssd_row_t));
            size_t ns = 0;
            const uint32_t qctx = qcnt[q];
            for (int r = 0; r < R && qctx; ++r) {
                const size_t rlen = (size_t)(ref->offs[r + 1] - ref->offs[r]);
                kssd_features_t f = feat_of(&c.ctx[(size_t)i * R + r], &c.obj[(size_t)i * R + r]);
                const uint32_t rctx = rcnt[r];
                if (kind == DETAIL_STREAM_ONE) {
                    /* compute_streamed_ref_row_one_qry, src/command_ani.c:2110-2201 */
                    if (rlen == 0 || rtotal[r] == 0)
                        continue;
                    const uint32_t need = kssd_af_needed_ctx(o, qctx, rtotal[r]);
                    if (rctx == 0 || f.XnY_ctx < (uint32_t)o->ctxcut || f.XnY_ctx < need)
                        continue;
                } else if (kind == DETAIL_STREAM_MULTI) {
                    /* src/command_ani.c:2933-2960 */
                    if (rctx == 0 || f.XnY_ctx < (uint32_t)o->ctxcut)
                        continue;
                } else {
                    /* comb_manysmall_...: src/command_ani.c:3945-3968 */
                    if (rctx == 0)
                        continue;
                    if (f.XnY_ctx < kssd_af_needed_ctx(o, qctx, rctx))
                        continue;
                }
                const double af_q = (double)f.XnY_ctx / (double)qctx;
                const double af_r = (double)f.XnY_ctx / (double)rctx;
                if (!kssd_af_pass(o, af_q, af_r))
                    continue;
                kssd_features_t t = f;
                t.X_ctx = qctx;
                const double bq = kssd_af_anib(&t, o->drfold);
                t = f;
                t.X_ctx = rctx;
                const double br = kssd_af_anib(&t, o->drfold);
                kssd_row_t row = kssd_make_row((uint32_t)r, &f, o, qctx, rctx, af_q, bq, af_r, br,
                                               qry->meta ? &qry->meta[q] : NULL, ref->meta ? &ref->meta[r] : NULL);
                if (kind != DETAIL_STREAM_MULTI && !kssd_row_passes_close_filter(&row, o))
                    continue;
                if (kind == DETAIL_HASH ? row.selected_ani <= o->anicut : row.selected_ani < o->anicut)
                    continue;
                surv[ns++] = row;
            }
            if (ns)
                qsort(surv, ns, sizeof *surv, kssd_cmp_row_desc);
            size_t out_n = ns;
            if (kind != DETAIL_HASH && o->ntop > 0 && (size_t)o->ntop < out_n)
                out_n = (size_t)o->ntop;
            if (o->estimate_coverage && kind != DETAIL_HASH && out_n) {
                const size_t qb = (size_t)(qry->offs[q] - qry->offs[0]);
                kssd_coverage_rows(qry->keys + qb, qab ? qab + qb : NULL, (size_t)(qry->offs[q + 1] - qry->offs[q]),
                                   ref->keys, ref->offs, cov.db.available ? &cov.db : NULL, qry->obj_bits, surv,
                                   out_n);
            }
            for (size_t k = 0; k < out_n; ++k)
                kssd_append_detail_row(&rows[i], o, qry->names[q], ref->names[surv[k].rn], &surv[k],
                                       anno_at(ref, surv[k].rn));
            free(surv);
        }
        for (int i = 0; i < nb; ++i) {
            write_buf(out, &rows[i]);
            kssd_buf_free(&rows[i]);
        }
        free(rows);
        free_counts(&c);
    }
    close_out(out);
    kssdgpu_index_free(ix);
    free(qab);
    cov_db_free(&cov);
    if (rtotal != rcnt)
        free(rtotal);
    free(qcnt);
    free(rcnt);
    kssd_sketch_free(qry);
    kssd_sketch_free(ref);
    return 0;
}

/* ------------------------------------------------------------------ dispatcher */

static void gen_index(const char *dir)
{
    kssd_sketch_t *s = load_sketch(dir, 0);
    if ((uint64_t)(s->offs[s->n] - s->offs[0]) >= 0xFFFFFFFFull)
        errx(EXIT_FAILURE, "gen_inverted_index4comblco():sketch_index maximun exceed UINT32_MAX");
    kssdgpu_index_t *ix = gpu_index_of_sketch(s);
    write_index_files(dir, ix, s->offs[s->n] - s->offs[0]);
    kssdgpu_index_free(ix);
    kssd_sketch_free(s);
}

/* run_sketch_ani, src/command_ani_wrapper.c:1082-1230 */
static int run_sketch_ani(void)
{
    kssd_ani_opt_t *o = &g.o;
    if ((g.unique_ctx || g.unique_report[0]) && !kssd_file_exists(g.refdir, "sortedcomb_ctxgid64obj32"))
        errx(EXIT_FAILURE, "unique-context options require an existing unfiltered reference inverted index; run "
                           "sketch -i on the reference sketch");
    if (o->unassembled && !o->afcut_set)
        o->afcut = 0.2f;
    kssd_sketch_stat_t qst;
    if (kssd_read_stat(g.qrydir, &qst))
        errx(EXIT_FAILURE, "%s", kssd_host_last_error());
    const int nq = qst.infile_num;
    o->drfold = qst.drfold;
    kssd_stat_bits(&qst, &o->ctx_bits, &o->obj_bits);
    const bool force = force_ref_index() || g.unique_ctx || g.unique_report[0];
    const int direct_n = o->fmt ? matrix_direct_threshold() : 0;
    const bool self = !g.refdir[0] || (o->fmt && same_file(g.refdir, g.qrydir));
    if (self) {
        if (!g.refdir[0] && o->fmt == 0)
            errx(EXIT_FAILURE, "one-sketch ANI detail output is not supported; use -m1 full matrix or -m2 triangle");
        if (o->fmt == 1 && (force || matrix_use_index(nq, nq, direct_n))) {
            if (force && !kssd_file_exists(g.qrydir, "sortedcomb_ctxgid64obj32"))
                errx(EXIT_FAILURE, "KSSD3A_FORCE_REF_INDEX requires reference index '%s/%s'", g.qrydir,
                     "sortedcomb_ctxgid64obj32");
            return run_self(0);
        }
        if (o->fmt == 2 && (force || matrix_use_index(nq, nq, direct_n)))
            return run_self(1);
        return run_self(2);
    }
    if (o->fmt == 2)
        errx(EXIT_FAILURE, "ANI triangle output requires one sketch or identical -r/-q sketches");
    kssd_sketch_stat_t rst;
    if (kssd_read_stat(g.refdir, &rst))
        errx(EXIT_FAILURE, "%s", kssd_host_last_error());
    const int nref = rst.infile_num;
    const bool small_stream = !force && o->fmt == 0 && nref > 0 && nq < nref;
    if (small_stream && nq == 1) {
        const char *lk = getenv("KSSD3A_QRAW_LOOKUP");
        if (lk && lk[0] && strcmp(lk, "sorted") && strcmp(lk, "fence") && strcmp(lk, "fencepost") && strcmp(lk, "hash"))
            errx(EXIT_FAILURE, "stream_ref_sketches_one_qraw_lookup(): invalid KSSD3A_QRAW_LOOKUP='%s' (use hash or sorted)", lk);
        return run_detail_scan(DETAIL_STREAM_ONE);
    }
    const char *multi = getenv("KSSD3A_QRAW_MULTI");
    if (o->fmt == 0 && nq > 1) {
        bool use_q = small_stream && nq <= env_int("KSSD3A_QRAW_MULTI_THRESHOLD", 20, 1, "positive integer");
        if (o->unassembled && !force && multi && multi[0]) {
            if (!strcmp(multi, "sortedindex"))
                use_q = true;
            else if (!strcmp(multi, "legacy") || !strcmp(multi, "refindex"))
                use_q = false;
            else
                errx(EXIT_FAILURE, "invalid KSSD3A_QRAW_MULTI='%s' (use sortedindex, refindex, or legacy)", multi);
        }
        if (use_q)
            return run_detail_scan(DETAIL_STREAM_MULTI);
    }
    const bool has_index = kssd_file_exists(g.refdir, "sortedcomb_ctxgid64obj32");
    if (o->fmt == 1) {
        if (force) {
            if (!has_index)
                errx(EXIT_FAILURE, "KSSD3A_FORCE_REF_INDEX requires reference index '%s/%s'", g.refdir,
                     "sortedcomb_ctxgid64obj32");
            return run_mem_eff();
        }
        if (matrix_use_index(nref, nq, direct_n)) {
            if (!has_index)
                gen_index(g.refdir);
            return run_mem_eff();
        }
    } else if (has_index)
        return run_mem_eff();
    const int auto_n = env_int("KSSD3A_AUTO_REF_INDEX_THRESHOLD", 100, 0, "non-negative integer; 0 disables");
    if (!o->v && !o->unassembled && o->fmt == 0 && auto_n > 0 && nref > auto_n) {
        gen_index(g.refdir);
        return run_mem_eff();
    }
    if (force)
        errx(EXIT_FAILURE, "KSSD3A_FORCE_REF_INDEX requires reference index '%s/%s'", g.refdir,
             "sortedcomb_ctxgid64obj32");
    if (o->fmt)
        return run_rect_matrix();
    return run_detail_scan(DETAIL_HASH);
}

/* ------------------------------------------------------------------ auto ANI on sequence inputs
 * FASTA/FASTQ inputs are sketched (on the GPU) into temporary sketch directories with
 * the parameters of the first sketch input, or the auto-sketch defaults, then merged
 * per side and counted like sketch inputs (src/command_ani_wrapper.c:842-1046,
 * 1275-1502). */

typedef struct path_list {
    char **v;
    int n, cap;
} path_list_t;

static void plist_push(path_list_t *l, const char *p)
{
    if (l->n == l->cap) {
        l->cap = l->cap ? 2 * l->cap : 8;
        l->v = realloc(l->v, (size_t)l->cap * sizeof(char *));
        if (!l->v)
            err(errno, "%s(): OOM path vector", "path_vec_push");
    }
    l->v[l->n] = strdup(p);
    if (!l->v[l->n])
        err(errno, "%s(): OOM path copy", "path_vec_push");
    l->n++;
}

static void read_path_list(const char *list_path, path_list_t *out, const char *option_name)
{
    FILE *list = fopen(list_path, "r");
    if (!list)
        err(errno, "can't open %s file %s", option_name, list_path);
    char *line = malloc(4096);
    int line_no = 0;
    while (fgets(line, 4096, list) != NULL) {
        line_no++;
        size_t len = strlen(line);
        if (len == 4095 && line[len - 1] != '\n' && line[len - 1] != '\r')
            errx(EXIT_FAILURE, "%s file %s line %d exceeds maximum line length %d", option_name, list_path, line_no,
                 4095);
        char *start = line;
        while (isspace((unsigned char)*start))
            start++;
        char *end = start + strlen(start);
        while (end > start && isspace((unsigned char)end[-1]))
            end--;
        *end = 0;
        if (!start[0])
            continue;
        if (strlen(start) >= PATHLEN)
            errx(EXIT_FAILURE, "%s file %s line %d path exceeds maximum length %d", option_name, list_path, line_no,
                 PATHLEN - 1);
        plist_push(out, start);
    }
    if (ferror(list))
        err(errno, "failed while reading %s file %s", option_name, list_path);
    free(line);
    fclose(list);
    if (out->n < 1)
        errx(EXIT_FAILURE, "%s file %s has no input paths", option_name, list_path);
}

static kssd_sketch_stat_t read_sketch_stat_or_die(const char *dir)
{
    kssd_sketch_stat_t st;
    if (kssd_read_stat(dir, &st))
        err(EINVAL, "%s(): %s", "read_lco_sketch_stat", kssd_host_last_error());
    return st;
}

static void validate_supported_auto_stat(const kssd_sketch_stat_t *st)
{
    /* src/command_ani_wrapper.c:918-949 */
    if (st->drfold < 0 || st->drfold > 32)
        errx(EXIT_FAILURE, "unsupported sketch drfold %d in first auto ANI sketch", st->drfold);
    if (st->klen > 32)
        errx(EXIT_FAILURE, "first auto ANI sketch has unsupported klen=%d; expected at most 32", st->klen);
    if (st->coden_len > 0) {
        if (st->coden_len != KSSD_NUM_CODENS)
            errx(EXIT_FAILURE, "first auto ANI sketch uses coden_len=%d, but this binary was built with NUM_CODENS=%d",
                 st->coden_len, KSSD_NUM_CODENS);
        const int expected = KSSD_NUM_CODENS < 11 ? 3 * KSSD_NUM_CODENS + 1 : 32;
        if (st->klen != expected)
            errx(EXIT_FAILURE, "first auto ANI sketch klen=%d is not compatible with coden_len=%d in this binary",
                 st->klen, st->coden_len);
    } else if (st->klen - 2 * (st->hclen + st->holen) < 0) {
        errx(EXIT_FAILURE, "first auto ANI sketch has invalid manual context-object lengths: klen=%d hclen=%d holen=%d",
             st->klen, st->hclen, st->holen);
    }
}

static bool same_auto_stat(const kssd_sketch_stat_t *a, const kssd_sketch_stat_t *b)
{
    return a->hash_id == b->hash_id && a->koc == b->koc && a->conflict == b->conflict &&
           a->coden_len == b->coden_len && a->klen == b->klen && a->hclen == b->hclen && a->holen == b->holen &&
           a->drfold == b->drfold;
}

static void validate_auto_inputs(const path_list_t *in, const kssd_sketch_stat_t *t)
{
    for (int i = 0; i < in->n; ++i) {
        if (!is_sketch_dir(in->v[i]))
            continue;
        kssd_sketch_stat_t st = read_sketch_stat_or_die(in->v[i]);
        if (!same_auto_stat(t, &st))
            errx(EXIT_FAILURE,
                 "%s sketch parameters do not match first auto ANI sketch "
                 "(hash_id %u/%u, koc %d/%d, conflict %d/%d, coden_len %d/%d, "
                 "klen %d/%d, hclen %d/%d, holen %d/%d, drfold %d/%d)",
                 in->v[i], st.hash_id, t->hash_id, st.koc, t->koc, st.conflict, t->conflict, st.coden_len,
                 t->coden_len, st.klen, t->klen, st.hclen, t->hclen, st.holen, t->holen, st.drfold, t->drfold);
    }
}

static kssd_sketch_stat_t default_auto_stat(void)
{
    return kssd_default_auto_stat(g.sketch_coden, g.sketch_hclen, g.sketch_holen, g.sketch_iolen, g.sketch_drfold,
                                  g.sketch_conflict, g.sketch_abundance);
}

static kssd_sketch_stat_t select_auto_template(const path_list_t *ref, const path_list_t *qry)
{
    const path_list_t *sides[2] = {ref, qry};
    for (int s = 0; s < 2; ++s)
        for (int i = 0; i < sides[s]->n; ++i)
            if (is_sketch_dir(sides[s]->v[i])) {
                kssd_sketch_stat_t st = read_sketch_stat_or_die(sides[s]->v[i]);
                validate_supported_auto_stat(&st);
                return st;
            }
    kssd_sketch_stat_t st = default_auto_stat();
    validate_supported_auto_stat(&st);
    return st;
}

/* Sketch options whose sketches need k-mer counts, read statistics, per-record
 * genomes or piped streams: not part of this build's sketcher. */
static void reject_unbuilt_sketch_options(const kssd_sketch_stat_t *t)
{
    const char *what = NULL;
    if (g.pipecmd[0])
        what = "--pipecmd";
    else if (g.sketch_split_mfa)
        what = "--splitmfa";
    else if (t->koc)
        what = "abundance (counting) sketches";
    else if (g.sketch_reads_qc)
        what = "--readsQC";
    else if (g.sketch_npercentile > 0.0)
        what = "--npercentile";
    else if (g.sketch_ncap > 0)
        what = "--ncap";
    else if (g.sketch_kmerocrs > 1)
        what = "--LstKmerOcrs above 1";
    if (what)
        errx(EXIT_FAILURE, "sequence inputs with %s are not supported by this build's sketcher; sketch them with "
                           "`kssd3a sketch` and pass the sketch directories", what);
}

static void sketch_arg_to_dir(const char *input, const kssd_sketch_stat_t *t, const char *outdir)
{
    reject_unbuilt_sketch_options(t);
    kssd_autosketch_opt_t ao;
    memset(&ao, 0, sizeof ao);
    ao.tmpl = *t;
    ao.asone = g.sketch_asone;
    ao.anno = g.sketch_anno;
    ao.threads = g.o.p > 0 ? g.o.p : 1;
    kssd_autosketch_to_dir(input, &ao, outdir);
}

static void prepare_side(const path_list_t *inputs, path_list_t *sketches, const char *prefix,
                         const kssd_sketch_stat_t *t, const char *tmp_root)
{
    for (int i = 0; i < inputs->n; ++i) {
        if (is_sketch_dir(inputs->v[i])) {
            plist_push(sketches, inputs->v[i]);
            continue;
        }
        char outdir[2 * PATHLEN];
        int w = snprintf(outdir, sizeof outdir, "%s/%sseq_%d", tmp_root, prefix, i);
        if (w < 0 || (size_t)w >= sizeof outdir)
            errx(EXIT_FAILURE, "auto ANI temporary output path is too long for %s", inputs->v[i]);
        sketch_arg_to_dir(inputs->v[i], t, outdir);
        plist_push(sketches, outdir);
    }
}

static void merge_side(const path_list_t *sketches, const char *outdir, char *dst, const char *label)
{
    const char *src = sketches->n == 1 ? sketches->v[0] : outdir;
    if (strlen(src) >= PATHLEN)
        errx(EXIT_FAILURE, "%s path is too long; maximum supported length is %d bytes", label, PATHLEN - 1);
    if (sketches->n > 1)
        kssd_merge_sketch_dirs(sketches->v, sketches->n, outdir);
    memcpy(dst, src, strlen(src) + 1);
}

static int count_stdin(const path_list_t *l)
{
    int c = 0;
    for (int i = 0; i < l->n; ++i)
        c += !strcmp(l->v[i], "-");
    return c;
}

static bool query_side_unassembled(const path_list_t *qry)
{
    for (int i = 0; i < qry->n; ++i) {
        const char *p = qry->v[i];
        if (is_sketch_dir(p))
            continue;
        if (strcmp(p, "-") && kssd_fastx_fmt(p) == KSSD_FMT_FASTQ)
            return true;
        if (g.sketch_conflict && (!strcmp(p, "-") || g.pipecmd[0]))
            return true;
    }
    return false;
}

static char g_tmp_root[PATHLEN];

static void remove_tmp_root(void)
{
    if (g_tmp_root[0])
        kssd_remove_tree(g_tmp_root);
}

static const char *make_tmp_root(const char *pattern)
{
    snprintf(g_tmp_root, sizeof g_tmp_root, "%s", pattern);
    if (!mkdtemp(g_tmp_root))
        err(errno, "%s(): mkdtemp", "run_auto_ani_from_sides");
    atexit(remove_tmp_root);
    return g_tmp_root;
}

static int run_auto_ani_from_sides(const path_list_t *ref, const path_list_t *qry)
{
    if (ref->n < 1)
        errx(EXIT_FAILURE, "auto ANI requires at least one reference input");
    if (qry->n < 1)
        errx(EXIT_FAILURE, "auto ANI requires at least one query input");
    if (count_stdin(ref) + count_stdin(qry) > 1)
        errx(EXIT_FAILURE, "stdin input '-' can be used only once in auto ANI");
    kssd_sketch_stat_t t = select_auto_template(ref, qry);
    validate_auto_inputs(ref, &t);
    validate_auto_inputs(qry, &t);
    const char *root = make_tmp_root("/tmp/kssd3a_ani_auto_XXXXXX");
    path_list_t rs = {0}, qs = {0};
    prepare_side(ref, &rs, "ref", &t, root);
    prepare_side(qry, &qs, "qry", &t, root);
    char rm[2 * PATHLEN], qm[2 * PATHLEN];
    snprintf(rm, sizeof rm, "%s/ref_merged", root);
    snprintf(qm, sizeof qm, "%s/qry_merged", root);
    merge_side(&rs, rm, g.refdir, "auto ANI reference sketch");
    merge_side(&qs, qm, g.qrydir, "auto ANI query sketch");
    if (query_side_unassembled(qry)) {
        g.o.unassembled = true;
        g.o.v = true;
    }
    return run_sketch_ani();
}

static int run_auto_positional_ani(void)
{
    if (g.nrem < 2)
        errx(EXIT_FAILURE, "auto ANI requires one reference input followed by at least one query input");
    path_list_t ref = {0}, qry = {0};
    plist_push(&ref, g.rem[0]);
    for (int i = 1; i < g.nrem; ++i)
        plist_push(&qry, g.rem[i]);
    return run_auto_ani_from_sides(&ref, &qry);
}

static int run_auto_list_ani(void)
{
    path_list_t ref = {0}, qry = {0};
    read_path_list(g.reflist, &ref, "--reflist");
    read_path_list(g.qrylist, &qry, "--qrylist");
    return run_auto_ani_from_sides(&ref, &qry);
}

static int run_direct_query_sequence_ani(bool force_raw, const char *option_name)
{
    /* src/command_ani_wrapper.c:1443-1502 */
    if (!is_sketch_dir(g.refdir))
        errx(EXIT_FAILURE,
             "%s sequence input requires -r/--ref to be a sketch directory; "
             "for direct reference sequence input use positional auto ANI",
             option_name);
    struct stat st;
    if (stat(g.qrydir, &st) == 0 && S_ISDIR(st.st_mode))
        errx(EXIT_FAILURE, "%s input '%s' is a directory but not a valid sketch", option_name, g.qrydir);
    kssd_sketch_stat_t t = read_sketch_stat_or_die(g.refdir);
    validate_supported_auto_stat(&t);
    if (force_raw || g.sketch_conflict)
        t.conflict = true;
    const char *root = make_tmp_root("/tmp/kssd3a_ani_query_XXXXXX");
    char out[2 * PATHLEN];
    int w = snprintf(out, sizeof out, "%s/qry_seq", root);
    if (w < 0 || (size_t)w >= sizeof out)
        errx(EXIT_FAILURE, "temporary %s sketch output path is too long", option_name);
    char input[PATHLEN];
    snprintf(input, sizeof input, "%s", g.qrydir);
    sketch_arg_to_dir(input, &t, out);
    if (strlen(out) >= sizeof g.qrydir)
        errx(EXIT_FAILURE, "temporary query sketch path is too long; maximum supported length is %zu bytes",
             sizeof g.qrydir - 1);
    memcpy(g.qrydir, out, strlen(out) + 1);
    g.o.unassembled = force_raw;
    if (force_raw)
        g.o.v = true;
    return run_sketch_ani();
}

static int cmd_ani(int argc, char **argv)
{
    memset(&g, 0, sizeof g);
    kssd_opt_defaults(&g.o);
    g.sketch_coden = true;
    g.sketch_hclen = 11;
    g.sketch_drfold = 8;
    g.sketch_kmerocrs = 1;
    argp_parse(&k_argp, argc, argv, ARGP_IN_ORDER, NULL, NULL);
    g.o.unique_ctx = g.unique_ctx;
    g.o.estimate_coverage = g.estimate_coverage;
    if (g.o.p < 1)
        g.o.p = 1;
    start_gpu_warmup();
    /* src/command_ani_wrapper.c:1519-1530 */
    if (g.reflist[0] || g.qrylist[0])
        run_auto_list_ani();
    else if (g.qrydir[0]) {
        if (!is_sketch_dir(g.qrydir))
            run_direct_query_sequence_ani(g.o.unassembled, g.o.unassembled ? "--qraw" : "-q/--query");
        else
            run_sketch_ani();
    } else if (g.nrem >= 2)
        run_auto_positional_ani();
    return 0;
}

/* ------------------------------------------------------------------ `kssd3a matrix`
 * Full and triangle reports of one sketch (matrix_write_indexed_self_matrix,
 * src/command_matrix.c:439-619) and the rectangular full report
 * (matrix_compute_dense, :258-315); options and validation of
 * src/command_matrix_wrapper.c:53-533.  The sparse graph formats (edges, clusters,
 * dedup-plan), --query-sketch-list and the legacy --ani matrix are not part of the
 * counting engine and are rejected. */

enum { MF_AUTO = 0, MF_FULL, MF_TRIANGLE, MF_EDGES, MF_CLUSTERS, MF_DEDUP };
enum { MM_MOE = 0, MM_NAIVE, MM_PDIST, MM_MASH, MM_AAF };

enum { MOP_SINGLE = 0, MOP_AND, MOP_OR };

typedef struct matrix_cli {
    int metric, metric_count, format, phylip, d, threads;
    int metrics[5], metric_op;   /* pairwise_metric_expr_t: up to 5 metrics joined by & or | */
    char metric_label[128];
    double e, diag, cut, max_afcut;
    bool cut_set, ani, max_afcut_set;
    uint32_t ctxcut, max_ctx_freq, min_votes, sample_step;
    int dedup_strategy;          /* 0 greedy, 1 full-linkage */
    char refdir[PATHLEN], qrydir[PATHLEN], qrylist[PATHLEN], outf[PATHLEN], gl[PATHLEN], idmap[PATHLEN];
    char edge_out[PATHLEN], keep_out[PATHLEN], remove_out[PATHLEN], keep_matrix_out[PATHLEN], keep_idmap[PATHLEN];
    int keep_matrix_fmt, dedup_seen, nrem;
    char **rem;
} matrix_cli_t;

static matrix_cli_t gm;

enum {
    MK_FORMAT = 900, MK_SPARSE, MK_CUT, MK_MAX_AFCUT, MK_CTXCUT, MK_DIAG_VALUE, MK_EDGE_OUT, MK_KEEP_OUT, MK_REMOVE_OUT,
    MK_MATRIX_FORMAT, MK_MATRIX_IDMAP, MK_KEEP_MATRIX_OUT, MK_KEEP_MATRIX_FORMAT, MK_KEEP_MATRIX_IDMAP,
    MK_MAX_CTX_FREQ, MK_MIN_VOTES, MK_SAMPLE_STEP, MK_QUERY_LIST, MK_PROGRESS, MK_DEDUP
};

static struct argp_option k_matrix_opts[] = {
    {"ref", 'r', "<DIR>", 0, "Reference sketches. Omit for triangle mode.", 9},
    {"query", 'q', "<DIR>", 0, "Query sketches.", 1},
    {"query-sketch-list", MK_QUERY_LIST, "<FILE>", 0,
     "One compatible -T query sketch directory per line; rectangular full matrix only.", 1},
    {"metric", 'm', "<METRIC>", 0, "ctx-moe, ctx-naive, p_dist, mash, or aaf; 0/1 alias mash/aaf. [ctx-naive]", 2},
    {"format", MK_FORMAT, "<FORMAT>", 0, "Report format: full, triangle, edges/sparse, clusters, or dedup-plan. "
                                         "[full for -r/-q; triangle for one sketch]", 2},
    {"sparse", MK_SPARSE, 0, 0, "Alias for --format sparse/edges; requires --cut.", 2},
    {"cut", MK_CUT, "<FLOAT>", 0, "Distance cutoff for sparse edge, cluster, and dedup-plan reports.", 3},
    {"dedup-strategy", MK_DEDUP, "<greedy|full-linkage>", 0,
     "Dedup-plan grouping strategy: greedy representative-neighbor or full-linkage clique. [greedy]", 3},
    {"control", 'c', "<FLOAT>", OPTION_HIDDEN, "Compatibility alias for --cut.", 3},
    {"max-afcut", MK_MAX_AFCUT, "<FLOAT>", 0,
     "Minimum max(Qry_align_fraction, Ref_align_fraction) for sparse edges. [0; 0.8 for dedup-plan]", 3},
    {"ctxcut", MK_CTXCUT, "<INT>", 0, "Minimum shared context count for sparse edges. [0]", 3},
    {"index-max-ctx-freq", MK_MAX_CTX_FREQ, "<INT>", 0,
     "Indexed sparse candidate mode: skip context groups above this frequency; 0 keeps all contexts. [256]", 3},
    {"index-min-votes", MK_MIN_VOTES, "<INT>", 0,
     "Indexed sparse candidate mode: exact-score pairs with at least this many candidate context votes. [1]", 3},
    {"index-sample-step", MK_SAMPLE_STEP, "<INT>", 0,
     "Indexed sparse candidate mode: use every Nth query context for nomination. [1]", 3},
    {"progress", MK_PROGRESS, "<auto|on|off>", 0, "Progress on stderr (accepted; no progress is printed).", 3},
    {"glist", 'g', "<FILE>", 0, "Sample output file for KSSD set grouping.", 4},
    {"outfile", 'o', "<FILE>", 0, "Matrix output file. [STDOUT]", 5},
    {"matrix-format", MK_MATRIX_FORMAT, "<tsv|phylip>", 0, "Output format for --format full. [tsv]", 5},
    {"matrix-idmap", MK_MATRIX_IDMAP, "<FILE>", 0, "With --matrix-format phylip, write short-ID to sample-name map.", 5},
    {"edge-out", MK_EDGE_OUT, "<FILE>", 0, "Optional sparse edge TSV for cluster/dedup-plan reports.", 5},
    {"keep-out", MK_KEEP_OUT, "<FILE>", 0, "Write one kept sample per line for dedup-plan reports.", 5},
    {"remove-out", MK_REMOVE_OUT, "<FILE>", 0, "Write one removed sample per line for dedup-plan reports.", 5},
    {"keep-matrix-out", MK_KEEP_MATRIX_OUT, "<FILE>", 0,
     "With dedup-plan, write a dense distance matrix for kept representatives.", 5},
    {"keep-matrix-format", MK_KEEP_MATRIX_FORMAT, "<tsv|phylip>", 0, "Output format for --keep-matrix-out. [tsv]", 5},
    {"keep-matrix-idmap", MK_KEEP_MATRIX_IDMAP, "<FILE>", 0,
     "With --keep-matrix-format phylip, write short-ID to sample-name map.", 5},
    {"threads", 'p', "<INT>", 0, "Number of host threads to use.", 6},
    {"diagonal", 'd', 0, 0, "Print diagonal values in triangle mode. [0]", 7},
    {"diagonal-value", MK_DIAG_VALUE, "<FLOAT>", 0, "Set diagonal value and enable diagonal output.", 7},
    {"exception", 'e', "<FLOAT>", 0, "Distance value to use when XnY == 0. [1]", 8},
    {"ani", 'n', 0, OPTION_HIDDEN, "Use context-object ANI mode.", 9},
    {0}};

static double parse_nonneg(struct argp_state *st, const char *name, const char *arg)
{
    char *end = NULL;
    errno = 0;
    double v = strtod(arg, &end);
    if (errno || end == arg || *end || !isfinite(v) || v < 0.0)
        argp_error(st, "%s requires a non-negative number", name);
    return v;
}

static bool matrix_metric_from(const char *arg, int *m)
{
    /* pairwise_metric_from_string, src/pairwise_graph.c:70-99 */
    static const struct { const char *name; int m; } names[] = {
        {"ctx-moe", MM_MOE}, {"moe", MM_MOE}, {"ctx-naive", MM_NAIVE}, {"naive", MM_NAIVE}, {"p_dist", MM_PDIST},
        {"pdist", MM_PDIST}, {"p-distance", MM_PDIST}, {"micro-obj", MM_PDIST}, {"micro_obj_rate", MM_PDIST},
        {"mash", MM_MASH}, {"mashd", MM_MASH}, {"0", MM_MASH}, {"aaf", MM_AAF}, {"aafd", MM_AAF}, {"1", MM_AAF}};
    for (size_t i = 0; i < sizeof names / sizeof names[0]; ++i)
        if (!strcmp(arg, names[i].name)) {
            *m = names[i].m;
            return true;
        }
    return false;
}

static error_t parse_matrix(int key, char *arg, struct argp_state *st)
{
    switch (key) {
    case 'm': {
        /* whitespace-free metric, or an A&B / A|B expression of such */
        char compact[128];
        size_t n = 0;
        for (const char *p = arg; *p; ++p)
            if (*p != ' ' && *p != '\t' && *p != '\n' && *p != '\r' && n + 1 < sizeof compact)
                compact[n++] = *p;
        compact[n] = '\0';
        int count = 0, m = 0;
        const bool has_and = strchr(compact, '&') != NULL, has_or = strchr(compact, '|') != NULL;
        bool ok = n > 0 && !(has_and && has_or);
        if (ok) {
            const char *delim = has_and ? "&" : (has_or ? "|" : "");
            if ((has_and || has_or) && (compact[0] == delim[0] || compact[n - 1] == delim[0] || strstr(compact, has_and ? "&&" : "||")))
                ok = false;
            char *save = NULL;
            for (char *tok = (has_and || has_or) ? strtok_r(compact, delim, &save) : compact; ok && tok;
                 tok = (has_and || has_or) ? strtok_r(NULL, delim, &save) : NULL) {
                int mm;
                if (count >= 5 || !matrix_metric_from(tok, &mm))
                    ok = false;
                else {
                    if (count == 0)
                        m = mm;
                    gm.metrics[count++] = mm;
                }
            }
        }
        if (!ok || count == 0)
            argp_error(st, "-m/--metric must be one metric such as ctx-naive, p_dist, mash, or aaf, or an expression "
                           "like 'ctx-naive&aaf' or 'ctx-moe|mash'");
        gm.metric = m;
        gm.metric_count = count;
        gm.metric_op = count == 1 ? MOP_SINGLE : (has_and ? MOP_AND : MOP_OR);
        /* pairwise_expr_append_label, src/pairwise_graph.c:154-170 */
        static const char *const names[] = {"ctx-moe", "ctx-naive", "p_dist", "mash", "aaf"};
        gm.metric_label[0] = '\0';
        for (int i = 0; i < count; ++i) {
            const size_t used = strlen(gm.metric_label);
            snprintf(gm.metric_label + used, sizeof gm.metric_label - used, "%s%s",
                     i == 0 ? "" : (gm.metric_op == MOP_AND ? "&" : "|"), names[gm.metrics[i]]);
        }
        break;
    }
    case MK_FORMAT:
        if (!strcmp(arg, "full") || !strcmp(arg, "matrix")) gm.format = MF_FULL;
        else if (!strcmp(arg, "triangle") || !strcmp(arg, "tri")) gm.format = MF_TRIANGLE;
        else if (!strcmp(arg, "edges") || !strcmp(arg, "edge") || !strcmp(arg, "sparse")) gm.format = MF_EDGES;
        else if (!strcmp(arg, "clusters") || !strcmp(arg, "cluster") || !strcmp(arg, "components")) gm.format = MF_CLUSTERS;
        else if (!strcmp(arg, "dedup-plan") || !strcmp(arg, "dedup")) gm.format = MF_DEDUP;
        else argp_error(st, "--format must be one of full, triangle, edges/sparse, clusters, or dedup-plan");
        break;
    case MK_SPARSE: gm.format = MF_EDGES; break;
    case 'c':
    case MK_CUT: gm.cut = parse_nonneg(st, "--cut", arg); gm.cut_set = true; break;
    case MK_MAX_AFCUT:
        gm.max_afcut = parse_double_range(st, "--max-afcut", arg, 0.0, 1.0);
        gm.max_afcut_set = true;
        break;
    case MK_CTXCUT: gm.ctxcut = (uint32_t)parse_int_range(st, "--ctxcut", arg, 0, INT32_MAX); break;
    case MK_MAX_CTX_FREQ:
        gm.max_ctx_freq = (uint32_t)parse_int_range(st, "--index-max-ctx-freq", arg, 0, INT32_MAX);
        break;
    case MK_MIN_VOTES: gm.min_votes = (uint32_t)parse_int_range(st, "--index-min-votes", arg, 1, INT32_MAX); break;
    case MK_SAMPLE_STEP:
        gm.sample_step = (uint32_t)parse_int_range(st, "--index-sample-step", arg, 1, INT32_MAX);
        break;
    case MK_PROGRESS:
        /* parse_matrix_progress, src/command_matrix_wrapper.c:216-228; progress itself is not printed */
        if (strcmp(arg, "auto") && strcmp(arg, "on") && strcmp(arg, "1") && strcmp(arg, "yes") && strcmp(arg, "off") &&
            strcmp(arg, "0") && strcmp(arg, "no"))
            argp_error(st, "--progress must be one of auto, on, or off");
        break;
    case MK_DEDUP:
        /* pairwise_dedup_strategy_from_string, src/pairwise_graph.c:118-140 */
        gm.dedup_seen = 1;
        if (!strcmp(arg, "greedy") || !strcmp(arg, "rep") || !strcmp(arg, "representative") ||
            !strcmp(arg, "rep-centric") || !strcmp(arg, "representative-centric"))
            gm.dedup_strategy = 0;
        else if (!strcmp(arg, "full") || !strcmp(arg, "full-linkage") || !strcmp(arg, "full_linkage") ||
                 !strcmp(arg, "complete") || !strcmp(arg, "complete-linkage") || !strcmp(arg, "complete_linkage") ||
                 !strcmp(arg, "clique"))
            gm.dedup_strategy = 1;
        else
            argp_error(st, "--dedup-strategy must be one of greedy, full-linkage, complete-linkage, or clique");
        break;
    case 'e': gm.e = parse_nonneg(st, "-e/--exception", arg); break;
    case 'p': gm.threads = parse_int_range(st, "-p/--threads", arg, 1, 65536); break;
    case 'q': copy_path(st, "-q/--query", gm.qrydir, arg); break;
    case MK_QUERY_LIST: copy_path(st, "--query-sketch-list", gm.qrylist, arg); break;
    case 'r': copy_path(st, "-r/--ref", gm.refdir, arg); break;
    case 'o': copy_path(st, "-o/--outfile", gm.outf, arg); break;
    case 'g': copy_path(st, "-g/--glist", gm.gl, arg); break;
    case MK_EDGE_OUT: copy_path(st, "--edge-out", gm.edge_out, arg); break;
    case MK_KEEP_OUT: copy_path(st, "--keep-out", gm.keep_out, arg); break;
    case MK_REMOVE_OUT: copy_path(st, "--remove-out", gm.remove_out, arg); break;
    case MK_MATRIX_FORMAT:
    case MK_KEEP_MATRIX_FORMAT: {
        /* parse_keep_matrix_format, src/command_matrix_wrapper.c:202-213 (both options) */
        int ph;
        if (!strcmp(arg, "tsv") || !strcmp(arg, "table")) ph = 0;
        else if (!strcmp(arg, "phylip") || !strcmp(arg, "phy") || !strcmp(arg, "fillip")) ph = 1;
        else { argp_error(st, "--keep-matrix-format must be one of tsv or phylip"); ph = 0; }
        if (key == MK_MATRIX_FORMAT) gm.phylip = ph; else gm.keep_matrix_fmt = ph;
        break;
    }
    case MK_MATRIX_IDMAP: copy_path(st, "--matrix-idmap", gm.idmap, arg); break;
    case MK_KEEP_MATRIX_OUT: copy_path(st, "--keep-matrix-out", gm.keep_matrix_out, arg); break;
    case MK_KEEP_MATRIX_IDMAP: copy_path(st, "--keep-matrix-idmap", gm.keep_idmap, arg); break;
    case 'd': gm.d = 1; break;
    case MK_DIAG_VALUE: gm.diag = parse_nonneg(st, "--diagonal-value", arg); gm.d = 1; break;
    case 'n': gm.ani = true; break;
    case ARGP_KEY_ARGS:
        gm.nrem = st->argc - st->next;
        gm.rem = st->argv + st->next;
        break;
    case ARGP_KEY_END: {
        /* src/command_matrix_wrapper.c:399-430 (the checks that concern full/triangle reports) */
        if (gm.qrydir[0] && gm.qrylist[0])
            argp_error(st, "-q/--query and --query-sketch-list are mutually exclusive");
        if (gm.qrylist[0] && gm.nrem > 0)
            argp_error(st, "--query-sketch-list cannot be combined with a positional sketch argument");
        if (!gm.qrydir[0] && !gm.qrylist[0] && gm.nrem == 1)
            copy_path(st, "sketch", gm.qrydir, gm.rem[0]);
        else if (gm.nrem > 0)
            argp_error(st, "matrix accepts at most one positional sketch argument; use -r/-q for rectangular reports");
        if (!gm.qrydir[0] && !gm.qrylist[0])
            argp_error(st, "missing sketch input; provide one sketch argument, -q/--query, or --query-sketch-list");
        if (gm.qrylist[0] && !gm.refdir[0])
            argp_error(st, "--query-sketch-list requires -r/--ref");
        if (gm.refdir[0] && gm.format == MF_TRIANGLE)
            argp_error(st, "--format triangle is only valid for one sketch");
        const int eff = gm.format != MF_AUTO ? gm.format : (gm.refdir[0] ? MF_FULL : MF_TRIANGLE);
        if (gm.metric_count > 1 && (eff == MF_FULL || eff == MF_TRIANGLE))
            argp_error(st, "combined --metric expressions are only valid for --sparse/--format edges, clusters, or "
                           "dedup-plan");
        if ((gm.format == MF_EDGES || gm.format == MF_CLUSTERS || gm.format == MF_DEDUP) && !gm.cut_set)
            argp_error(st, "--sparse/--format edges, clusters, or dedup-plan requires --cut");
        if ((gm.format == MF_CLUSTERS || gm.format == MF_DEDUP) && gm.refdir[0])
            argp_error(st, "--format clusters/dedup-plan requires one sketch, not -r/-q");
        if ((gm.keep_out[0] || gm.remove_out[0] || gm.keep_matrix_out[0] || gm.keep_idmap[0]) && eff != MF_DEDUP)
            argp_error(st, "--keep-out/--remove-out/--keep-matrix-out/--keep-matrix-idmap require --format dedup-plan");
        if (gm.dedup_seen && eff != MF_DEDUP)
            argp_error(st, "--dedup-strategy requires --format dedup-plan");
        if (gm.phylip && eff != MF_FULL)
            argp_error(st, "--matrix-format phylip requires --format full");
        if (gm.phylip && gm.refdir[0])
            argp_error(st, "--matrix-format phylip requires one square sketch, not -r/-q");
        if (gm.qrylist[0] && (eff != MF_FULL || gm.ani))
            argp_error(st, "--query-sketch-list currently supports rectangular --format full without --ani");
        if (gm.idmap[0] && !gm.phylip)
            argp_error(st, "--matrix-idmap requires --matrix-format phylip");
        if (gm.keep_matrix_fmt && !gm.keep_matrix_out[0])
            argp_error(st, "--keep-matrix-format requires --keep-matrix-out");
        if (gm.keep_idmap[0] && !gm.keep_matrix_out[0])
            argp_error(st, "--keep-matrix-idmap requires --keep-matrix-out");
        if (gm.keep_idmap[0] && !gm.keep_matrix_fmt)
            argp_error(st, "--keep-matrix-idmap requires --keep-matrix-format phylip");
        /* output files must all differ, in the reference's order of checks */
        static const struct { int a, b; const char *msg; } diff[] = {
            {3, 4, "--keep-out and --remove-out must be different files"},
            {3, 0, "--keep-out must differ from --outfile"},
            {4, 0, "--remove-out must differ from --outfile"},
            {5, 0, "--keep-matrix-out must differ from --outfile"},
            {1, 0, "--matrix-idmap must differ from --outfile"},
            {2, 0, "--edge-out must differ from --outfile"},
            {3, 2, "--keep-out must differ from --edge-out"},
            {4, 2, "--remove-out must differ from --edge-out"},
            {5, 2, "--keep-matrix-out must differ from --edge-out"},
            {5, 3, "--keep-matrix-out must differ from --keep-out"},
            {5, 4, "--keep-matrix-out must differ from --remove-out"},
            {6, 0, "--keep-matrix-idmap must differ from --outfile"},
            {6, 2, "--keep-matrix-idmap must differ from --edge-out"},
            {6, 3, "--keep-matrix-idmap must differ from --keep-out"},
            {6, 4, "--keep-matrix-idmap must differ from --remove-out"},
            {6, 5, "--keep-matrix-idmap must differ from --keep-matrix-out"},
            {1, 2, "--matrix-idmap must differ from --edge-out"},
            {1, 3, "--matrix-idmap must differ from --keep-out"},
            {1, 4, "--matrix-idmap must differ from --remove-out"},
            {1, 5, "--matrix-idmap must differ from --keep-matrix-out"},
            {1, 6, "--matrix-idmap must differ from --keep-matrix-idmap"},
        };
        const char *files[7] = {gm.outf, gm.idmap, gm.edge_out, gm.keep_out, gm.remove_out, gm.keep_matrix_out,
                                gm.keep_idmap};
        for (size_t i = 0; i < sizeof diff / sizeof diff[0]; ++i)
            if (files[diff[i].a][0] && files[diff[i].b][0] && !strcmp(files[diff[i].a], files[diff[i].b]))
                argp_error(st, "%s", diff[i].msg);
        break;
    }
    default:
        return ARGP_ERR_UNKNOWN;
    }
    return 0;
}

static struct argp k_matrix_argp = {k_matrix_opts, parse_matrix, 0,
                                    "\nReport pairwise sketch distance matrices; shared-context counting on the GPU.",
                                    NULL, NULL, NULL};

/* matrix_kput_fixed6, src/command_matrix.c:103-124 */
static void put_fixed6(kssd_buf_t *b, double v)
{
    if (!isfinite(v) || v > 900000000000.0 || v < -900000000000.0) {
        kssd_buf_printf(b, "%lf", v);
        return;
    }
    if (v < 0.0) {
        kssd_buf_putc(b, '-');
        v = -v;
    }
    const uint64_t scaled = (uint64_t)(v * 1000000.0 + 0.5);
    uint32_t frac = (uint32_t)(scaled % 1000000ULL);
    kssd_buf_printf(b, "%ld.", (long)(scaled / 1000000ULL));
    char f6[7];
    for (int i = 5; i >= 0; --i) {
        f6[i] = (char)('0' + frac % 10);
        frac /= 10;
    }
    f6[6] = '\0';
    kssd_buf_puts(b, f6);
}

/* matrix_scale_fixed6 / matrix_kput_scaled6, src/command_matrix.c:126-149 */
static uint32_t scale_u6(double v)
{
    if (!isfinite(v))
        v = 1.0;
    if (v < 0.0)
        v = 0.0;
    if (v > 4294.0)
        v = 4294.0;
    return (uint32_t)(v * 1000000.0 + 0.5);
}

static void put_u6(kssd_buf_t *b, uint32_t scaled)
{
    char f6[8];
    uint32_t frac = scaled % 1000000U;
    for (int i = 5; i >= 0; --i) {
        f6[i] = (char)('0' + frac % 10);
        frac /= 10;
    }
    f6[6] = '\0';
    kssd_buf_printf(b, "%u.%s", scaled / 1000000U, f6);
}

/* matrix_context_metric_distance, src/command_matrix.c:400-424 */
static double matrix_metric_distance(int metric, const kssd_features_t *f, uint32_t qc, uint32_t rc,
                                     const kssd_ani_opt_t *o)
{
    kssd_features_t t = *f;
    switch (metric) {
    case MM_NAIVE: return kssd_naive_dist(&t);
    case MM_MOE: return kssd_lm3ways_dist(&t, o->drfold);
    case MM_PDIST: return kssd_p_dist(&t, o->obj_bits);
    case MM_MASH: return kssd_mashD((uint32_t)(o->ctx_bits / 2), rc, qc, f->XnY_ctx);
    default: return kssd_aafD((uint32_t)(o->ctx_bits / 2), rc, qc, f->XnY_ctx);
    }
}

/* matrix_context_feature_value, src/command_matrix.c:621-661: the metric expression
 * over clamped distances (& keeps the largest, | the smallest) */
static double matrix_context_value(const kssd_features_t *f, uint32_t qc, uint32_t rc, const kssd_ani_opt_t *o)
{
    if (f->XnY_ctx == 0 || qc == 0 || rc == 0)
        return gm.e;
    double selected = 0.0;
    for (int i = 0; i < gm.metric_count; ++i) {
        double d = matrix_metric_distance(gm.metrics[i], f, qc, rc, o);
        if (!isfinite(d))
            return gm.e;
        if (d < 0.0) d = 0.0;
        if (d > 1.0) d = 1.0;
        if (i == 0)
            selected = d;
        else if (gm.metric_op == MOP_AND ? d > selected : d < selected)
            selected = d;
    }
    return selected;
}

/* pairwise_eval_arrays distances, src/pairwise_graph.c:13-49,301-360 */
static double clean_dist(double d) { return !isfinite(d) ? 1.0 : (d < 0.0 ? 0.0 : d); }

static double pair_metric_distance(int metric, const kssd_features_t *f, uint32_t qc, uint32_t rc,
                                   const kssd_ani_opt_t *o)
{
    kssd_features_t t = *f;
    const int k = o->ctx_bits > 0 ? o->ctx_bits / 2 : 32;
    switch (metric) {
    case MM_MASH: {
        const double denom = (double)qc + (double)rc - (double)f->XnY_ctx;
        if (denom <= 0.0) return 1.0;
        const double j = (double)f->XnY_ctx / denom, tr = (2.0 * j) / (1.0 + j);
        if (tr <= 0.0) return 1.0;
        return clean_dist(-log(tr) / (double)k);
    }
    case MM_AAF: {
        const uint32_t m = qc < rc ? qc : rc;
        if (m == 0) return 1.0;
        const double c = (double)f->XnY_ctx / (double)m;
        if (c <= 0.0) return 1.0;
        return clean_dist(-log(c) / (double)k);
    }
    case MM_NAIVE: return clean_dist(kssd_naive_dist(&t));
    case MM_PDIST: return clean_dist(kssd_p_dist(&t, o->obj_bits));
    default: return clean_dist(kssd_lm3ways_dist(&t, o->drfold));
    }
}

/* pairwise_eval_t (src/pairwise_graph.h) of one (query, reference) pair */
typedef struct pair_eval {
    double distance, similarity, af_qry, af_ref, max_af;
    uint32_t xny, n_diff_obj, n_diff_obj_section, n_mut2_ctx;
    bool valid;
} pair_eval_t;

/* pairwise_eval_arrays + pairwise_eval_expr_merge (src/pairwise_graph.c:301-360,417-446):
 * the features are the pair's shared-context counters; the metric expression keeps the
 * largest (&) or smallest (|) distance, the first of equals. */
static pair_eval_t pair_eval(const kssd_features_t *f, uint32_t qc, uint32_t rc, size_t qlen, size_t rlen,
                             const kssd_ani_opt_t *o)
{
    pair_eval_t e = {.distance = 1.0};
    if (qlen == 0 || rlen == 0)
        return e;
    e.xny = f->XnY_ctx;
    e.n_diff_obj = f->N_diff_obj;
    e.n_diff_obj_section = f->N_diff_obj_section;
    e.n_mut2_ctx = f->N_mut2_ctx;
    e.af_qry = qc > 0 ? (double)f->XnY_ctx / (double)qc : 0.0;
    e.af_ref = rc > 0 ? (double)f->XnY_ctx / (double)rc : 0.0;
    e.max_af = e.af_qry > e.af_ref ? e.af_qry : e.af_ref;
    if (f->XnY_ctx == 0)
        return e;
    double sel = 1.0;
    for (int i = 0; i < gm.metric_count; ++i) {
        const double d = pair_metric_distance(gm.metrics[i], f, qc, rc, o);
        if (i == 0 || (gm.metric_op == MOP_AND ? d > sel : d < sel))
            sel = d;
    }
    e.distance = sel;
    e.similarity = 1.0 - sel;
    e.valid = true;
    return e;
}

static double matrix_pair_value(const kssd_features_t *f, uint32_t qc, uint32_t rc, size_t qlen, size_t rlen,
                                const kssd_ani_opt_t *o)
{
    const pair_eval_t e = pair_eval(f, qc, rc, qlen, rlen, o);
    return e.valid ? e.distance : gm.e;
}

static void matrix_glist(const kssd_sketch_t *s)
{
    if (!gm.gl[0])
        return;
    FILE *f = fopen(gm.gl, "w");
    if (!f)
        err(errno, "matrix_write_glist(): Failed to open file:%s\n", gm.gl);
    for (int i = 0; i < s->n; ++i)
        fprintf(f, "%d\t%s\n", i + 1, s->names[i]);
    fclose(f);
}

static int matrix_self(int fmt)
{
    kssd_sketch_t *s = load_sketch(gm.qrydir, 0);
    init_bits(s);
    const int n = s->n;
    g.o.ignoreconflict = false;
    g.o.p = gm.threads;
    kssdgpu_ctx_mut2_t *lc = NULL;
    kssdgpu_obj_section_t *lo = NULL;
    self_lower_counts(s, gm.qrydir, kssd_file_exists(gm.qrydir, "sortedcomb_ctxgid64obj32"), false, &lc, &lo);
    uint32_t *cnt = sample_ctx_counts(s, s->stat.conflict, false);
    const size_t cells = (size_t)n * (n - 1) / 2;
    double *v = malloc(cells * sizeof(double) + 8);
    if (!v)
        err(EXIT_FAILURE, "OOM matrix values");
#pragma omp parallel for schedule(dynamic, 16) num_threads(gm.threads)
    for (int q = 1; q < n; ++q) {
        const size_t base = (size_t)q * (q - 1) / 2;
        for (int r = 0; r < q; ++r) {
            kssd_features_t f = feat_of(&lc[base + r], &lo[base + r]);
            v[base + r] = matrix_context_value(&f, cnt[q], cnt[r], &g.o);
        }
    }
    free(lc);
    free(lo);
    FILE *out = open_out(gm.outf);
    kssd_buf_t h = {0};
    if (fmt == MF_FULL) {
        if (gm.phylip) {
            if (gm.idmap[0]) {
                /* matrix_write_full_matrix_idmap, src/command_matrix.c:365-379 */
                FILE *im = open_out(gm.idmap);
                fputs("id\tsample\n", im);
                for (int i = 0; i < n; ++i)
                    fprintf(im, "S%09d\t%s\n", i + 1, s->names[i]);
                if (im != stdout)
                    fclose(im);
            }
            kssd_buf_printf(&h, "%d\n", n);
        } else {
            for (int r = 0; r < n; ++r) {
                kssd_buf_putc(&h, '\t');
                kssd_buf_puts(&h, s->names[r]);
            }
            kssd_buf_putc(&h, '\n');
        }
        write_buf(out, &h);
        kssd_buf_free(&h);
    }
    const uint32_t diag_u6 = scale_u6(gm.diag);
    const int chunk = 256;
    for (int q0 = 0; q0 < n; q0 += chunk) {
        const int nb = n - q0 < chunk ? n - q0 : chunk;
        kssd_buf_t *rows = calloc((size_t)nb, sizeof(kssd_buf_t));
#pragma omp parallel for schedule(dynamic, 1) num_threads(gm.threads)
        for (int i = 0; i < nb; ++i) {
            const int q = q0 + i;
            kssd_buf_t *b = &rows[i];
            if (fmt == MF_FULL && gm.phylip) {
                char id[16];
                snprintf(id, sizeof id, "S%09d", q + 1);
                kssd_buf_printf(b, "%-10s", id);
            } else {
                kssd_buf_puts(b, s->names[q]);
            }
            if (fmt == MF_FULL) {
                for (int r = 0; r < n; ++r) {
                    uint32_t u = diag_u6;
                    if (q > r)
                        u = scale_u6(v[(size_t)q * (q - 1) / 2 + r]);
                    else if (q < r)
                        u = scale_u6(v[(size_t)r * (r - 1) / 2 + q]);
                    kssd_buf_putc(b, gm.phylip ? ' ' : '\t');
                    put_u6(b, u);
                }
            } else {
                for (int r = 0; r < q; ++r) {
                    kssd_buf_putc(b, '\t');
                    put_fixed6(b, v[(size_t)q * (q - 1) / 2 + r]);
                }
                if (gm.d) {
                    kssd_buf_putc(b, '\t');
                    put_fixed6(b, gm.diag);
                }
            }
            kssd_buf_putc(b, '\n');
        }
        for (int i = 0; i < nb; ++i) {
            write_buf(out, &rows[i]);
            kssd_buf_free(&rows[i]);
        }
        free(rows);
    }
    close_out(out);
    matrix_glist(s);
    free(v);
    free(cnt);
    kssd_sketch_free(s);
    return 0;
}

/* matrix_load_query_sketch_list (src/command_matrix.c:1350-1450): the listed sketch
 * directories (one per line; blank lines and # comments skipped), compatible with the
 * first, concatenated into one query sketch */
static char *trim_line(char *line)
{
    while (*line && isspace((unsigned char)*line))
        ++line;
    char *end = line + strlen(line);
    while (end > line && isspace((unsigned char)end[-1]))
        *--end = '\0';
    return line;
}

static kssd_sketch_t *load_query_list(const char *list_path)
{
    FILE *fp = fopen(list_path, "r");
    if (!fp)
        err(errno, "open failed for %s", list_path);
    kssd_sketch_t **parts = NULL;
    size_t np = 0, cap = 0, samples = 0, entries = 0;
    char *line = NULL;
    size_t lcap = 0;
    while (getline(&line, &lcap, fp) >= 0) {
        char *dir = trim_line(line);
        if (!*dir || *dir == '#')
            continue;
        kssd_sketch_t *part = load_sketch(dir, 0);
        if (np) {
            const kssd_sketch_stat_t *e = &parts[0]->stat, *a = &part->stat;
            if (e->hash_id != a->hash_id || e->koc != a->koc || e->conflict != a->conflict ||
                e->coden_len != a->coden_len || e->klen != a->klen || e->hclen != a->hclen || e->holen != a->holen ||
                e->drfold != a->drfold)
                errx(EINVAL, "--query-sketch-list entry is incompatible with the first entry: %s", dir);
        }
        if (np == cap) {
            cap = cap ? cap * 2 : 16;
            parts = realloc(parts, cap * sizeof(*parts));
            if (!parts)
                err(EXIT_FAILURE, "realloc query sketch list");
        }
        parts[np++] = part;
        samples += (size_t)part->n;
        entries += (size_t)(part->offs[part->n] - part->offs[0]);
    }
    free(line);
    fclose(fp);
    if (np == 0)
        errx(EINVAL, "no query sketch directories listed in %s", list_path);
    if (samples > (size_t)INT_MAX)
        errx(EOVERFLOW, "--query-sketch-list is too large");
    kssd_sketch_t *m = calloc(1, sizeof *m);
    if (!m)
        err(EXIT_FAILURE, "allocate merged query sketch");
    m->stat = parts[0]->stat;
    m->stat.infile_num = (int32_t)samples;
    m->n = (int)samples;
    m->obj_bits = parts[0]->obj_bits;
    m->ctx_bits = parts[0]->ctx_bits;
    m->names = malloc((samples ? samples : 1) * KSSD_PATHLEN);
    m->keys = malloc((entries ? entries : 1) * sizeof(uint64_t));
    m->offs = calloc(samples + 1, sizeof(uint64_t));
    if (!m->names || !m->keys || !m->offs)
        err(EXIT_FAILURE, "allocate merged query sketch payload");
    size_t so = 0, eo = 0;
    for (size_t p = 0; p < np; ++p) {
        const kssd_sketch_t *part = parts[p];
        const size_t pe = (size_t)(part->offs[part->n] - part->offs[0]);
        for (int i = 0; i < part->n; ++i) {
            memcpy(m->names[so + (size_t)i], part->names[i], KSSD_PATHLEN);
            m->offs[so + (size_t)i + 1] = eo + (part->offs[i + 1] - part->offs[0]);
        }
        if (pe)
            memcpy(m->keys + eo, part->keys, pe * sizeof(uint64_t));
        so += (size_t)part->n;
        eo += pe;
        kssd_sketch_free(parts[p]);
    }
    free(parts);
    return m;
}

static int matrix_rect(void)
{
    kssd_sketch_t *ref = load_sketch(gm.refdir, 0);
    kssd_sketch_t *qry = gm.qrylist[0] ? load_query_list(gm.qrylist) : load_sketch(gm.qrydir, 0);
    if (ref->stat.hash_id != qry->stat.hash_id)
        errx(EXIT_FAILURE, "pairwise_check_compatible(): ref hash_id %u != qry %u", ref->stat.hash_id,
             qry->stat.hash_id);
    init_bits(ref);
    g.o.p = gm.threads;
    const bool same = !gm.qrylist[0] && !strcmp(gm.refdir, gm.qrydir);
    uint32_t *qc = sample_ctx_counts(qry, qry->stat.conflict, false);
    uint32_t *rc = sample_ctx_counts(ref, ref->stat.conflict, false);
    kssdgpu_index_t *ix = gpu_index_of_sketch(ref);
    FILE *out = open_out(gm.outf);
    kssd_buf_t h = {0};
    for (int r = 0; r < ref->n; ++r) {
        kssd_buf_putc(&h, '\t');
        kssd_buf_puts(&h, ref->names[r]);
    }
    kssd_buf_putc(&h, '\n');
    write_buf(out, &h);
    kssd_buf_free(&h);
    const int R = ref->n, B = block_for(R, qry->n);
    for (int q0 = 0; q0 < qry->n; q0 += B) {
        const int nb = qry->n - q0 < B ? qry->n - q0 : B;
        counts_t c = count_queries(ix, R, qry, q0, nb, 0);
        kssd_buf_t *rows = calloc((size_t)nb, sizeof(kssd_buf_t));
#pragma omp parallel for schedule(dynamic, 1) num_threads(gm.threads)
        for (int i = 0; i < nb; ++i) {
            const int q = q0 + i;
            const size_t qlen = (size_t)(qry->offs[q + 1] - qry->offs[q]);
            kssd_buf_puts(&rows[i], qry->names[q]);
            for (int r = 0; r < R; ++r) {
                double v = gm.diag;
                if (!(same && q == r)) {
                    kssd_features_t f = feat_of(&c.ctx[(size_t)i * R + r], &c.obj[(size_t)i * R + r]);
                    v = matrix_pair_value(&f, qc[q], rc[r], qlen, (size_t)(ref->offs[r + 1] - ref->offs[r]), &g.o);
                }
                kssd_buf_printf(&rows[i], "\t%lf", v);
            }
            kssd_buf_putc(&rows[i], '\n');
        }
        for (int i = 0; i < nb; ++i) {
            write_buf(out, &rows[i]);
            kssd_buf_free(&rows[i]);
        }
        free(rows);
        free_counts(&c);
    }
    close_out(out);
    kssdgpu_index_free(ix);
    free(qc);
    free(rc);
    kssd_sketch_free(ref);
    kssd_sketch_free(qry);
    return 0;
}

/* ------------------------------------------------------------------ sparse reports
 *
 * `kssd3a matrix --format edges|clusters|dedup-plan` (src/command_matrix.c:660-1300,
 * src/pairwise_graph.c:518-1316).  Every pair's features come from the GPU self join
 * (one sketch) or block counts (-r/-q); with an index file and a conflict-free sketch
 * the reference nominates candidate pairs by context votes (GPU: kssdgpu_self_votes) and
 * reports edges row by row in the order its scan touches them; the union-find
 * components, greedy and full-linkage dedup plans and every report are host code.
 */

typedef struct sp_edge {
    int a, b;
} sp_edge_t;

typedef struct sp_edges {
    sp_edge_t *e;
    size_t n, cap;
} sp_edges_t;

static void sp_push(sp_edges_t *l, int a, int b)
{
    if (l->n == l->cap) {
        l->cap = l->cap ? l->cap * 2 : 1024;
        l->e = realloc(l->e, l->cap * sizeof(sp_edge_t));
        if (!l->e)
            err(EXIT_FAILURE, "OOM edge list");
    }
    l->e[l->n++] = (sp_edge_t){a, b};
}

/* matrix_print_edge_header / matrix_print_edge, src/command_matrix.c:87-101 */
static void print_edge_header(FILE *f)
{
    fputs("Qry\tRef\tDistance\tSimilarity\tMetric\tXnY_ctx\tQry_align_fraction\tRef_align_fraction\tmax_AF\t"
          "N_diff_obj\tN_diff_obj_section\tN_mut2_ctx\n",
          f);
}

static void print_edge(FILE *f, const char *q, const char *r, const pair_eval_t *e)
{
    fprintf(f, "%s\t%s\t%.12g\t%.12g\t%s\t%u\t%.12g\t%.12g\t%.12g\t%u\t%u\t%u\n", q, r, e->distance, e->similarity,
            gm.metric_label, e->xny, e->af_qry, e->af_ref, e->max_af, e->n_diff_obj, e->n_diff_obj_section,
            e->n_mut2_ctx);
}

/* pairwise_eval_passes_edge and the reject counters around it (src/pairwise_graph.c:
 * 518-530,1229-1245): 0 = no distance edge, 1 = shared-context reject, 2 = align-fraction
 * reject, 3 = accepted */
static int edge_class(const pair_eval_t *e)
{
    if (!e->valid || e->distance >= gm.cut)
        return 0;
    if (e->xny < gm.ctxcut)
        return 1;
    if (e->max_af < gm.max_afcut)
        return 2;
    return 3;
}

/* one sketch: lower-triangle counters, per-sample context counts */
typedef struct sp_self {
    const kssd_sketch_t *s;
    const kssdgpu_ctx_mut2_t *lc;
    const kssdgpu_obj_section_t *lo;
    const uint32_t *cnt;
} sp_self_t;

static size_t sp_len(const kssd_sketch_t *s, int i) { return (size_t)(s->offs[i + 1] - s->offs[i]); }

/* pairwise_eval_expr_samples(metric, sketch, qry, sketch, ref) from the pair's cell */
static pair_eval_t sp_eval(const sp_self_t *c, int qry, int ref)
{
    const int hi = qry > ref ? qry : ref, lo = qry > ref ? ref : qry;
    const size_t cell = (size_t)hi * (size_t)(hi - 1) / 2 + (size_t)lo;
    const kssd_features_t f = feat_of(&c->lc[cell], &c->lo[cell]);
    return pair_eval(&f, c->cnt[qry], c->cnt[ref], sp_len(c->s, qry), sp_len(c->s, ref), &g.o);
}

/* ---- sample quality (src/pairwise_graph.c:532-603) and representative rules
 * (src/command_matrix.c:151-246) */

static bool sp_meta_valid(const kssd_sketch_t *s, int i)
{
    return s->meta && i >= 0 && i < s->n && s->meta[i].meta_fmt_version == 1 && s->meta[i].total_length_bp > 0;
}

static double finite_or(double v, double fb) { return isfinite(v) ? v : fb; }

static int positive_lower_u32_cmp(uint32_t a, uint32_t b)
{
    if (a == b) return 0;
    if (a == 0) return -1;
    if (b == 0) return 1;
    return a < b ? 1 : -1;
}

/* > 0: a is the better representative */
static int sp_quality_cmp(const kssd_sketch_t *s, int a, int b)
{
    if (a == b)
        return 0;
    const bool ra = sp_meta_valid(s, a), rb = sp_meta_valid(s, b);
    if (ra != rb)
        return ra ? 1 : -1;
    if (ra && rb) {
        const kssd_infile_meta_t *ma = &s->meta[a], *mb = &s->meta[b];
        const bool fa = ma->infile_fmt == 1, fb = mb->infile_fmt == 1;
        if (fa != fb)
            return fa ? 1 : -1;
        const double aa = finite_or((double)ma->asm_level, -1.0), ab = finite_or((double)mb->asm_level, -1.0);
        if (aa != ab)
            return aa > ab ? 1 : -1;
        if (ma->total_length_bp != mb->total_length_bp)
            return ma->total_length_bp > mb->total_length_bp ? 1 : -1;
        const int rc = positive_lower_u32_cmp(ma->record_count, mb->record_count);
        if (rc)
            return rc;
        if (ma->median_length_bp != mb->median_length_bp)
            return ma->median_length_bp > mb->median_length_bp ? 1 : -1;
        const double ca = finite_or((double)ma->length_cv, INFINITY), cb = finite_or((double)mb->length_cv, INFINITY);
        if (ca != cb)
            return ca < cb ? 1 : -1;
    }
    const size_t ea = sp_len(s, a), eb = sp_len(s, b);
    if (ea != eb)
        return ea > eb ? 1 : -1;
    return a < b ? 1 : -1;
}

static const kssd_sketch_t *g_sp_sketch;
static int sp_order_cmp(const void *x, const void *y)
{
    return -sp_quality_cmp(g_sp_sketch, *(const int *)x, *(const int *)y);
}

/* samples best first (the comparison is a total order, so any sort gives the reference's) */
static int *sp_quality_order(const kssd_sketch_t *s)
{
    int *o = malloc((size_t)(s->n ? s->n : 1) * sizeof(int));
    if (!o)
        err(EXIT_FAILURE, "OOM quality order");
    for (int i = 0; i < s->n; ++i)
        o[i] = i;
    g_sp_sketch = s;
    qsort(o, (size_t)s->n, sizeof(int), sp_order_cmp);
    return o;
}

static const char *sp_rep_rule(const kssd_sketch_t *s, int sample, int rep)
{
    if (sample == rep)
        return "self";
    const bool sv = sp_meta_valid(s, sample), rv = sp_meta_valid(s, rep);
    if (sv != rv)
        return rv ? "valid_metadata" : "sample_valid_metadata";
    if (sv && rv) {
        const kssd_infile_meta_t *sm = &s->meta[sample], *rm = &s->meta[rep];
        const bool sf = sm->infile_fmt == 1, rf = rm->infile_fmt == 1;
        if (sf != rf)
            return rf ? "fasta_input" : "sample_fasta_input";
        if (sm->asm_level != rm->asm_level)
            return rm->asm_level > sm->asm_level ? "higher_asm_level" : "sample_higher_asm_level";
        if (sm->total_length_bp != rm->total_length_bp)
            return rm->total_length_bp > sm->total_length_bp ? "longer_total_length" : "sample_longer_total_length";
        if (sm->record_count != rm->record_count) {
            if (sm->record_count == 0)
                return "sample_missing_record_count";
            if (rm->record_count == 0)
                return "rep_missing_record_count";
            return rm->record_count < sm->record_count ? "fewer_records" : "sample_fewer_records";
        }
        if (sm->median_length_bp != rm->median_length_bp)
            return rm->median_length_bp > sm->median_length_bp ? "longer_median_length"
                                                               : "sample_longer_median_length";
        if (sm->length_cv != rm->length_cv)
            return rm->length_cv < sm->length_cv ? "lower_length_cv" : "sample_lower_length_cv";
    }
    const size_t se = sp_len(s, sample), re = sp_len(s, rep);
    if (se != re)
        return re > se ? "larger_sketch_entries" : "sample_larger_sketch_entries";
    return rep < sample ? "earlier_sample_order" : "sample_earlier_sample_order";
}

static void sp_print_meta(FILE *f, const kssd_sketch_t *s, int i)
{
    if (!sp_meta_valid(s, i)) {
        fputs("\tNA\tNA\tNA\tNA\tNA\tNA", f);
        return;
    }
    const kssd_infile_meta_t *m = &s->meta[i];
    fprintf(f, "\t%s\t%.6g\t%" PRIu64 "\t%u\t%u\t%.6g",
            m->infile_fmt == 1 ? "FASTA" : m->infile_fmt == 2 ? "FASTQ" : "NA", (double)m->asm_level,
            m->total_length_bp, m->record_count, m->median_length_bp, (double)m->length_cv);
}

/* ---- components and dedup plans (src/pairwise_graph.c:605-975) */

typedef struct sp_comp {
    int n;
    int *parent, *size, *rep;
    uint8_t *rank;
    bool *removed;
} sp_comp_t;

static void sp_comp_init(sp_comp_t *c, int n)
{
    c->n = n;
    c->parent = malloc((size_t)(n ? n : 1) * sizeof(int));
    c->size = calloc((size_t)(n ? n : 1), sizeof(int));
    c->rep = malloc((size_t)(n ? n : 1) * sizeof(int));
    c->rank = calloc((size_t)(n ? n : 1), 1);
    c->removed = calloc((size_t)(n ? n : 1), sizeof(bool));
    if (!c->parent || !c->size || !c->rep || !c->rank || !c->removed)
        err(EXIT_FAILURE, "OOM component bookkeeping");
    for (int i = 0; i < n; ++i) {
        c->parent[i] = i;
        c->rep[i] = -1;
    }
}

static void sp_comp_free(sp_comp_t *c)
{
    free(c->parent);
    free(c->size);
    free(c->rep);
    free(c->rank);
    free(c->removed);
}

static int sp_find(int *parent, int x)
{
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

static void sp_union(sp_comp_t *c, int a, int b)
{
    int ra = sp_find(c->parent, a), rb = sp_find(c->parent, b);
    if (ra == rb)
        return;
    if (c->rank[ra] < c->rank[rb])
        c->parent[ra] = rb;
    else if (c->rank[ra] > c->rank[rb])
        c->parent[rb] = ra;
    else {
        c->parent[rb] = ra;
        ++c->rank[ra];
    }
}

/* pairwise_component_result_finalize: sizes, best-quality representative per component */
static void sp_comp_finalize(sp_comp_t *c, const kssd_sketch_t *s)
{
    for (int i = 0; i < c->n; ++i) {
        const int r = sp_find(c->parent, i);
        c->parent[i] = r;
        ++c->size[r];
    }
    for (int i = 0; i < c->n; ++i) {
        const int r = c->parent[i];
        if (c->rep[r] < 0 || sp_quality_cmp(s, i, c->rep[r]) > 0)
            c->rep[r] = i;
    }
    for (int i = 0; i < c->n; ++i)
        c->removed[i] = i != c->rep[c->parent[i]];
}

/* pairwise_greedy_dedup_from_edges: best sample first claims all its unclaimed neighbours */
static void sp_dedup_greedy(sp_comp_t *c, const kssd_sketch_t *s, const sp_edges_t *edges)
{
    const int n = c->n;
    size_t *off = calloc((size_t)n + 1, sizeof(size_t));
    if (!off)
        err(EXIT_FAILURE, "OOM dedup graph");
    for (size_t e = 0; e < edges->n; ++e) {
        ++off[edges->e[e].a + 1];
        ++off[edges->e[e].b + 1];
    }
    for (int i = 0; i < n; ++i)
        off[i + 1] += off[i];
    int *adj = malloc((off[n] ? off[n] : 1) * sizeof(int));
    size_t *cur = malloc(((size_t)n + 1) * sizeof(size_t));
    if (!adj || !cur)
        err(EXIT_FAILURE, "OOM dedup adjacency");
    memcpy(cur, off, ((size_t)n + 1) * sizeof(size_t));
    for (size_t e = 0; e < edges->n; ++e) {
        adj[cur[edges->e[e].a]++] = edges->e[e].b;
        adj[cur[edges->e[e].b]++] = edges->e[e].a;
    }
    int *order = sp_quality_order(s);
    for (int oi = 0; oi < n; ++oi) {
        const int rep = order[oi];
        if (c->removed[rep])
            continue;
        c->parent[rep] = rep;
        c->rep[rep] = rep;
        c->size[rep] = 1;
        for (size_t k = off[rep]; k < off[rep + 1]; ++k) {
            const int x = adj[k];
            if (x == rep || c->removed[x])
                continue;
            c->removed[x] = true;
            c->parent[x] = rep;
            c->rep[x] = rep;
            ++c->size[rep];
        }
    }
    for (int i = 0; i < n; ++i)
        if (c->rep[i] < 0) {
            c->rep[i] = i;
            c->size[i] = 1;
        }
    free(order);
    free(cur);
    free(adj);
    free(off);
}

/* pairwise_complete_linkage_dedup_from_edges: in quality order, a representative takes
 * every unassigned sample linked to all members taken so far */
static void sp_dedup_complete(sp_comp_t *c, const kssd_sketch_t *s, const sp_edges_t *edges)
{
    const int n = c->n;
    const size_t words = ((size_t)n * (size_t)n + 63) / 64;
    uint64_t *bits = calloc(words ? words : 1, sizeof(uint64_t));
    int *members = malloc((size_t)(n ? n : 1) * sizeof(int));
    bool *assigned = calloc((size_t)(n ? n : 1), sizeof(bool));
    if (!bits || !members || !assigned)
        err(EXIT_FAILURE, "OOM full-linkage dedup");
    for (size_t e = 0; e < edges->n; ++e) {
        const size_t a = (size_t)edges->e[e].a, b = (size_t)edges->e[e].b;
        bits[(a * n + b) >> 6] |= 1ull << ((a * n + b) & 63);
        bits[(b * n + a) >> 6] |= 1ull << ((b * n + a) & 63);
    }
    int *order = sp_quality_order(s);
    for (int oi = 0; oi < n; ++oi) {
        const int rep = order[oi];
        if (assigned[rep])
            continue;
        assigned[rep] = true;
        c->parent[rep] = rep;
        c->rep[rep] = rep;
        c->size[rep] = 1;
        members[0] = rep;
        int mn = 1;
        for (int ci = 0; ci < n; ++ci) {
            const int x = order[ci];
            if (x == rep || assigned[x])
                continue;
            bool all = true;
            for (int mi = 0; mi < mn && all; ++mi) {
                const size_t pos = (size_t)x * n + (size_t)members[mi];
                all = (bits[pos >> 6] >> (pos & 63)) & 1ull;
            }
            if (!all)
                continue;
            c->removed[x] = true;
            assigned[x] = true;
            c->parent[x] = rep;
            c->rep[x] = rep;
            ++c->size[rep];
            members[mn++] = x;
        }
    }
    for (int i = 0; i < n; ++i)
        if (c->rep[i] < 0) {
            c->rep[i] = i;
            c->size[i] = 1;
        }
    free(order);
    free(assigned);
    free(members);
    free(bits);
}

/* ---- reports (src/command_matrix.c:317-380,801-939,1056-1123) */

static FILE *sp_open(const char *path)
{
    FILE *f = path[0] ? fopen(path, "w") : stdout;
    if (!f)
        err(errno, "matrix_open_output(): %s", path);
    return f;
}

static void sp_close(FILE *f)
{
    if (f != stdout)
        fclose(f);
    else
        fflush(f);
}

/* kept representatives' dense matrix from the lower counters (the indexed form,
 * matrix_write_keep_matrix_indexed) */
static void sp_keep_matrix(const sp_self_t *c, const sp_comp_t *comp)
{
    if (!gm.keep_matrix_out[0])
        return;
    const kssd_sketch_t *s = c->s;
    int *kept = malloc((size_t)(s->n ? s->n : 1) * sizeof(int));
    if (!kept)
        err(EXIT_FAILURE, "OOM kept samples");
    int kn = 0;
    for (int i = 0; i < s->n; ++i)
        if (!comp->removed[i])
            kept[kn++] = i;
    if (gm.keep_idmap[0]) {
        FILE *im = sp_open(gm.keep_idmap);
        fputs("id\tsample\n", im);
        for (int i = 0; i < kn; ++i)
            fprintf(im, "S%09d\t%s\n", i + 1, s->names[kept[i]]);
        sp_close(im);
    }
    FILE *f = sp_open(gm.keep_matrix_out);
    if (gm.keep_matrix_fmt) {
        fprintf(f, "%d\n", kn);
    } else {
        for (int k = 0; k < kn; ++k)
            fprintf(f, "\t%s", s->names[kept[k]]);
        fputc('\n', f);
    }
    for (int qi = 0; qi < kn; ++qi) {
        const int q = kept[qi];
        if (gm.keep_matrix_fmt) {
            char id[16];
            snprintf(id, sizeof id, "S%09d", qi + 1);
            fprintf(f, "%-10s", id);
        } else {
            fputs(s->names[q], f);
        }
        for (int k = 0; k < kn; ++k) {
            const int r = kept[k];
            double v = gm.diag;
            if (q != r) {
                const int hi = q > r ? q : r, lo = q > r ? r : q;
                const size_t cell = (size_t)hi * (size_t)(hi - 1) / 2 + (size_t)lo;
                const kssd_features_t ft = feat_of(&c->lc[cell], &c->lo[cell]);
                v = matrix_context_value(&ft, c->cnt[q], c->cnt[r], &g.o);
            }
            if (gm.keep_matrix_fmt)
                fprintf(f, " %.12g", v);
            else
                fprintf(f, "\t%lf", v);
        }
        fputc('\n', f);
    }
    sp_close(f);
    free(kept);
}

/* matrix_write_component_report */
static void sp_component_report(const sp_self_t *c, sp_comp_t *comp, bool dedup)
{
    const kssd_sketch_t *s = c->s;
    const int n = s->n;
    int *cid = calloc((size_t)(n ? n : 1), sizeof(int));
    if (!cid)
        err(EXIT_FAILURE, "OOM cluster ids");
    int next = 1;
    for (int i = 0; i < n; ++i) {
        const int root = sp_find(comp->parent, i);
        if (!cid[root])
            cid[root] = next++;
    }
    FILE *out = sp_open(gm.outf);
    FILE *keep = dedup && gm.keep_out[0] ? sp_open(gm.keep_out) : NULL;
    FILE *rem = dedup && gm.remove_out[0] ? sp_open(gm.remove_out) : NULL;
    if (dedup)
        fputs("sample\tcomponent_id\taction\trepresentative\treason\trep_rule\tcomponent_size\tsample_sketch_entries\t"
              "rep_sketch_entries\tsample_fmt\tsample_asm_level\tsample_total_length_bp\tsample_record_count\t"
              "sample_median_length_bp\tsample_length_cv\trep_fmt\trep_asm_level\trep_total_length_bp\t"
              "rep_record_count\trep_median_length_bp\trep_length_cv\n",
              out);
    else
        fputs("sample\tcluster_id\tcomponent_size\trepresentative\n", out);
    for (int i = 0; i < n; ++i) {
        const int root = sp_find(comp->parent, i);
        const int rep = comp->rep[root];
        if (dedup) {
            const bool single = comp->size[root] == 1, kept = i == rep;
            if (kept && keep)
                fprintf(keep, "%s\n", s->names[i]);
            if (!kept && rem)
                fprintf(rem, "%s\n", s->names[i]);
            fprintf(out, "%s\tcluster_%06d\t%s\t%s\t%s\t%s\t%d\t%" PRIu64 "\t%" PRIu64, s->names[i], cid[root],
                    kept ? "keep" : "remove", s->names[rep],
                    single ? "singleton" : (kept ? "best_representative" : "duplicate"), sp_rep_rule(s, i, rep),
                    comp->size[root], (uint64_t)sp_len(s, i), (uint64_t)sp_len(s, rep));
            sp_print_meta(out, s, i);
            sp_print_meta(out, s, rep);
            fputc('\n', out);
        } else {
            fprintf(out, "%s\tcluster_%06d\t%d\t%s\n", s->names[i], cid[root], comp->size[root], s->names[rep]);
        }
    }
    sp_close(out);
    if (keep)
        sp_close(keep);
    if (rem)
        sp_close(rem);
    sp_keep_matrix(c, comp);
    free(cid);
}

/* ---- one sketch */

typedef struct sp_touch {
    uint32_t first;
    int r;
} sp_touch_t;

static int matrix_sparse_self(int fmt)
{
    const bool comps = fmt == MF_CLUSTERS || fmt == MF_DEDUP, dedup = fmt == MF_DEDUP;
    /* matrix_parse_flags_for_format: component reports read the input metadata */
    kssd_sketch_t *s = load_sketch(gm.qrydir, comps ? 2u : 0u);
    init_bits(s);
    g.o.p = gm.threads;
    g.o.ignoreconflict = false;
    if (dedup && !gm.max_afcut_set)
        gm.max_afcut = 0.8;
    const int n = s->n;
    const size_t cells = (size_t)n * (size_t)(n > 0 ? n - 1 : 0) / 2;
    /* exact features of every pair: the self join over the sketch's own index */
    kssdgpu_ctx_mut2_t *lc = malloc(cells * sizeof(*lc) + 8);
    kssdgpu_obj_section_t *lo = malloc(cells * sizeof(*lo) + 8);
    if (!lc || !lo)
        err(EXIT_FAILURE, "OOM lower triangle");
    kssdgpu_index_t *ix = gpu_index_of_sketch(s);
    if (cells)
        gpu_check(kssdgpu_self_lower(ix, 0, lc, lo), "device self join");
    uint32_t *cnt = sample_ctx_counts(s, s->stat.conflict, false);
    const sp_self_t c = {s, lc, lo, cnt};
    /* matrix_can_use_sorted_index: conflict-free sketch with an index file */
    const bool indexed = !s->stat.conflict && kssd_file_exists(gm.qrydir, "sortedcomb_ctxgid64obj32");
    FILE *edge_out = NULL;
    if (comps) {
        if (gm.edge_out[0]) {
            edge_out = sp_open(gm.edge_out);
            print_edge_header(edge_out);
        }
    } else {
        edge_out = sp_open(gm.outf);
        print_edge_header(edge_out);
    }
    sp_comp_t comp;
    sp_comp_init(&comp, n);
    sp_edges_t edges = {0};
    if (indexed) {
        /* pairwise_indexed_self_scan: votes over the index file's records */
        size_t nrec = 0;
        kssd_index_rec_t *rec = kssd_index_load(gm.qrydir, &nrec);
        if (!rec)
            errx(EXIT_FAILURE, "%s", kssd_host_last_error());
        if (nrec != (size_t)(s->offs[n] - s->offs[0]))
            errx(EINVAL, "pairwise_indexed_self_scan(): %s/sortedcomb_ctxgid64obj32 has %zu records, expected %llu",
                 gm.qrydir, nrec, (unsigned long long)(s->offs[n] - s->offs[0]));
        kssdgpu_index_t *vix = ix;
        if (records_checksum(rec, nrec) != sketch_checksum(s))
            gpu_check(kssdgpu_index_from_records(rec, nrec, n, s->obj_bits, 0, &vix), "device index");
        free(rec);
        uint32_t *votes = malloc(cells * sizeof(uint32_t) + 4), *first = malloc(cells * sizeof(uint32_t) + 4);
        if (!votes || !first)
            err(EXIT_FAILURE, "OOM votes");
        if (cells)
            gpu_check(kssdgpu_self_votes(vix, s->keys, s->offs, gm.max_ctx_freq, gm.sample_step, votes, first),
                      "device votes");
        if (vix != ix)
            kssdgpu_index_free(vix);
        /* rows in order; within a row, edges in the order the scan first touched them */
        sp_edges_t *rows = calloc((size_t)(n ? n : 1), sizeof(sp_edges_t));
        if (!rows)
            err(EXIT_FAILURE, "OOM rows");
#pragma omp parallel for schedule(dynamic, 16) num_threads(gm.threads)
        for (int q = 1; q < n; ++q) {
            const size_t base = (size_t)q * (size_t)(q - 1) / 2;
            sp_touch_t *t = NULL;
            size_t tn = 0, tc = 0;
            for (int r = 0; r < q; ++r) {
                if (!votes[base + r] || votes[base + r] < gm.min_votes)
                    continue;
                const pair_eval_t e = sp_eval(&c, q, r);
                if (edge_class(&e) != 3)
                    continue;
                if (tn == tc) {
                    tc = tc ? tc * 2 : 16;
                    t = realloc(t, tc * sizeof(sp_touch_t));
                    if (!t)
                        err(EXIT_FAILURE, "OOM row edges");
                }
                t[tn++] = (sp_touch_t){first[base + r], r};
            }
            /* by first touch, then gid (the order of a context group's postings) */
            for (size_t i = 1; i < tn; ++i) {
                const sp_touch_t x = t[i];
                size_t j = i;
                while (j > 0 && (t[j - 1].first > x.first || (t[j - 1].first == x.first && t[j - 1].r > x.r))) {
                    t[j] = t[j - 1];
                    --j;
                }
                t[j] = x;
            }
            for (size_t i = 0; i < tn; ++i)
                sp_push(&rows[q], q, t[i].r);
            free(t);
        }
        for (int q = 1; q < n; ++q) {
            for (size_t i = 0; i < rows[q].n; ++i) {
                const int a = rows[q].e[i].a, b = rows[q].e[i].b;
                if (comps && !dedup)
                    sp_union(&comp, a, b);
                if (dedup)
                    sp_push(&edges, a, b);
                if (edge_out) {
                    const pair_eval_t e = sp_eval(&c, a, b);
                    print_edge(edge_out, s->names[a], s->names[b], &e);
                }
            }
            free(rows[q].e);
        }
        free(rows);
        free(votes);
        free(first);
    } else if (!comps) {
        /* matrix_compute_edges on one sketch: reference samples outer, later queries inner */
        for (int rn = 0; rn < n; ++rn)
            for (int qn = rn + 1; qn < n; ++qn) {
                const pair_eval_t e = sp_eval(&c, qn, rn);
                if (edge_class(&e) == 3)
                    print_edge(edge_out, s->names[qn], s->names[rn], &e);
            }
    } else {
        /* pairwise_build_components / pairwise_collect_dedup_edges: all pairs i < j */
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) {
                const pair_eval_t e = sp_eval(&c, i, j);
                if (edge_class(&e) != 3)
                    continue;
                if (dedup)
                    sp_push(&edges, i, j);
                else
                    sp_union(&comp, i, j);
                if (edge_out)
                    print_edge(edge_out, s->names[i], s->names[j], &e);
            }
    }
    if (edge_out)
        sp_close(edge_out);
    if (comps) {
        if (dedup) {
            if (gm.dedup_strategy)
                sp_dedup_complete(&comp, s, &edges);
            else
                sp_dedup_greedy(&comp, s, &edges);
        } else {
            sp_comp_finalize(&comp, s);
        }
        sp_component_report(&c, &comp, dedup);
    }
    matrix_glist(s);
    free(edges.e);
    sp_comp_free(&comp);
    kssdgpu_index_free(ix);
    free(cnt);
    free(lc);
    free(lo);
    kssd_sketch_free(s);
    return 0;
}

/* ---- -r/-q edges (matrix_compute_edges): reference samples outer, queries inner */

typedef struct sp_redge {
    int rn, qn;
    pair_eval_t e;
} sp_redge_t;

static int matrix_sparse_rect(void)
{
    kssd_sketch_t *ref = load_sketch(gm.refdir, 0);
    kssd_sketch_t *qry = load_sketch(gm.qrydir, 0);
    if (ref->stat.hash_id != qry->stat.hash_id)
        errx(EXIT_FAILURE, "pairwise_check_compatible(): ref hash_id %u != qry %u", ref->stat.hash_id,
             qry->stat.hash_id);
    init_bits(ref);
    g.o.p = gm.threads;
    const bool same = !strcmp(gm.refdir, gm.qrydir);
    uint32_t *qc = sample_ctx_counts(qry, qry->stat.conflict, false);
    uint32_t *rc = sample_ctx_counts(ref, ref->stat.conflict, false);
    kssdgpu_index_t *ix = gpu_index_of_sketch(ref);
    const int R = ref->n, B = block_for(R, qry->n);
    sp_redge_t *all = NULL;
    size_t an = 0, ac = 0;
    for (int q0 = 0; q0 < qry->n; q0 += B) {
        const int nb = qry->n - q0 < B ? qry->n - q0 : B;
        counts_t cts = count_queries(ix, R, qry, q0, nb, 0);
        for (int i = 0; i < nb; ++i) {
            const int q = q0 + i;
            for (int r = 0; r < R; ++r) {
                if (same && q <= r)
                    continue;
                const kssdgpu_ctx_mut2_t *cc = &cts.ctx[(size_t)i * R + r];
                if (!cc->num_ctx)
                    continue;
                const kssd_features_t f = feat_of(cc, &cts.obj[(size_t)i * R + r]);
                const pair_eval_t e = pair_eval(&f, qc[q], rc[r], sp_len(qry, q), sp_len(ref, r), &g.o);
                if (edge_class(&e) != 3)
                    continue;
                if (an == ac) {
                    ac = ac ? ac * 2 : 1024;
                    all = realloc(all, ac * sizeof(sp_redge_t));
                    if (!all)
                        err(EXIT_FAILURE, "OOM edges");
                }
                all[an++] = (sp_redge_t){r, q, e};
            }
        }
        free_counts(&cts);
    }
    /* counting sort by reference sample; queries already ascend within one */
    size_t *start = calloc((size_t)R + 1, sizeof(size_t));
    sp_redge_t *sorted = malloc((an ? an : 1) * sizeof(sp_redge_t));
    if (!start || !sorted)
        err(EXIT_FAILURE, "OOM edge order");
    for (size_t i = 0; i < an; ++i)
        ++start[all[i].rn + 1];
    for (int r = 0; r < R; ++r)
        start[r + 1] += start[r];
    for (size_t i = 0; i < an; ++i)
        sorted[start[all[i].rn]++] = all[i];
    FILE *out = sp_open(gm.outf);
    print_edge_header(out);
    for (size_t i = 0; i < an; ++i)
        print_edge(out, qry->names[sorted[i].qn], ref->names[sorted[i].rn], &sorted[i].e);
    sp_close(out);
    free(sorted);
    free(start);
    free(all);
    kssdgpu_index_free(ix);
    free(qc);
    free(rc);
    kssd_sketch_free(ref);
    kssd_sketch_free(qry);
    return 0;
}

static int cmd_matrix(int argc, char **argv)
{
    memset(&gm, 0, sizeof gm);
    memset(&g, 0, sizeof g);
    kssd_opt_defaults(&g.o);
    gm.metric = MM_NAIVE;
    gm.metric_count = 1;
    gm.metrics[0] = MM_NAIVE;
    gm.metric_op = MOP_SINGLE;
    snprintf(gm.metric_label, sizeof gm.metric_label, "ctx-naive");
    gm.threads = 1;
    gm.e = 1.0;
    gm.max_ctx_freq = 256;
    gm.min_votes = 1;
    gm.sample_step = 1;
    argp_parse(&k_matrix_argp, argc, argv, ARGP_IN_ORDER, NULL, NULL);
    const int fmt = gm.format != MF_AUTO ? gm.format : (gm.refdir[0] ? MF_FULL : MF_TRIANGLE);
    if (gm.refdir[0] && gm.ani)
        errx(EXIT_FAILURE, "the legacy --ani matrix is not supported by this build; use `kssd3a ani --format matrix`");
    if ((!gm.qrylist[0] && !is_sketch_dir(gm.qrydir)) || (gm.refdir[0] && !is_sketch_dir(gm.refdir)))
        errx(EXIT_FAILURE, "matrix inputs must be sketch directories");
    if (gm.qrylist[0]) {
        /* compute_matrix_query_list: rectangular full matrix against the listed queries */
        start_gpu_warmup();
        return matrix_rect();
    }
    start_gpu_warmup();
    if (!gm.refdir[0])
        return (fmt == MF_EDGES || fmt == MF_CLUSTERS || fmt == MF_DEDUP) ? matrix_sparse_self(fmt) : matrix_self(fmt);
    if (fmt == MF_EDGES)
        return matrix_sparse_rect();
    if (fmt != MF_FULL)
        errx(EINVAL, "compute_matrix(): --format clusters, dedup-plan, and triangle require one sketch");
    return matrix_rect();
}

int main(int argc, char **argv)
{
    setvbuf(stdout, NULL, _IOFBF, 1 << 20);
    phase("start");
    if (argc < 2) {
        fprintf(stderr, "Usage: %s ani [OPTION...]\n", argv[0]);
        return 64;
    }
    if (!strcmp(argv[1], "ani"))
        return cmd_ani(argc - 1, argv + 1);
    if (!strcmp(argv[1], "matrix"))
        return cmd_matrix(argc - 1, argv + 1);
    if (!strcmp(argv[1], "--version") || !strcmp(argv[1], "-V")) {
        printf("%s\n", argp_program_version);
        return 0;
    }
    fprintf(stderr, "%s: subcommand '%s' is not part of the counting engine; use the reference binary\n", argv[0],
            argv[1]);
    return 64;
}
