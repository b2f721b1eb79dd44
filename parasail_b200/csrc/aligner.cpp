/*
 * aligner.cpp -- parasail_b200_aligner: the reference's aligner driver
 * (apps/parasail_aligner.cpp of jeffdaily/parasail v2.6.2) over this
 * library's batch API.
 *
 * Same command line, defaults, checks, messages and output files: sequences
 * from a FASTA/FASTQ file (and an optional query file) are packed into one
 * '$'-separated text, candidate pairs come from the exact-match filter
 * (pairs sharing a substring of -c characters) or from all pairs, every
 * pair is aligned by the chosen function, and the results are written as
 * CSV (basic or statistics), edges, a graph, or -- for trace functions --
 * EMBOSS, SSW or SAM text. What changes is where the work runs:
 *   - the text is resident on the GPU as a packed sequence set
 *     (parasail_b200_seqdb_create: 2/5/8 bits a residue);
 *   - the filter runs on the GPU (parasail_b200_candidate_pairs) instead of
 *     a suffix array walked on one core;
 *   - pairs are aligned in memory-budgeted batches, each one GPU pipeline
 *     (parasail_b200_batch_pairs_seqdb, parasail_b200_nw_banded_batch,
 *     parasail_b200_batch_pairs_trace) instead of an OpenMP loop of
 *     per-pair calls; the output of a batch is written by a second thread
 *     while the next batch aligns.
 * The option -t (threads) is accepted and ignored. PSSM matrices are not
 * supported (the batch kernels take square matrices).
 */
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <poll.h>
#include <sys/time.h>
#include <unistd.h>

#include "parasail.h"
#include "parasail/io.h"
#include "parasail_b200.h"

namespace {

typedef std::pair<int, int> Pair;

const char *g_progname = "parasail_aligner";

void print_help(int status)
{
    fprintf(stderr,
            "\nusage: %s [-a funcname] [-c cutoff] [-x] [-e gap_extend] [-o gap_open] [-m matrix] [-t threads] "
            "[-d] [-M match] [-X mismatch] [-k band size (for nw_banded)] [-l AOL] [-s SIM] [-i OS] [-v] [-V] "
            "-f file [-q query_file] [-g output_file] [-O output_format {EMBOSS,SAM,SAMH,SSW}] [-b batch_size] "
            "[-r memory_budget] [-C] [-A alphabet_aliases] \n\n",
            g_progname);
    fprintf(stderr,
            "Defaults:\n"
            "        funcname: sw_stats_striped_16\n"
            "          cutoff: 7, must be >= 1, exact match length cutoff\n"
            "              -x: if present, don't use suffix array filter\n"
            "      gap_extend: 1, must be >= 0\n"
            "        gap_open: 10, must be >= 0\n"
            "          matrix: blosum62\n"
            "              -d: if present, assume DNA alphabet ACGT\n"
            "           match: 1, must be >= 0\n"
            "        mismatch: 0, must be >= 0\n"
            "         threads: accepted and ignored; the work runs on the GPU\n"
            "             AOL: 80, must be 0 <= AOL <= 100, percent alignment length\n"
            "             SIM: 40, must be 0 <= SIM <= 100, percent exact matches\n"
            "              OS: 30, must be 0 <= OS <= 100, percent optimal score\n"
            "                                              over self score\n"
            "              -v: verbose output, report input parameters and timing\n"
            "              -V: verbose memory output, report memory use\n"
            "            file: no default, must be in FASTA format\n"
            "      query_file: no default, must be in FASTA format\n"
            "     output_file: parasail.csv\n"
            "   output_format: no default, must be one of {EMBOSS,SAM,SAMH,SSW}\n"
            "      batch_size: 0 (calculate based on memory budget),\n"
            "                  how many alignments before writing output\n"
            "   memory_budget: 4GB of device memory for each batch\n"
            "              -C: if present, use case sensitive alignments, matrices, etc.\n"
            "alphabet_aliases: traceback will treat these pairs of characters as matches,\n"
            "                  for example, 'TU' for one pair, or multiple pairs as 'XYab'\n");
    exit(status);
}

double now()
{
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + tv.tv_usec * 1e-6;
}

/* data waiting on standard input within 100 ms (apps/parasail_aligner.cpp:365-374) */
bool stdin_has_data()
{
    struct pollfd fd;
    fd.fd = 0;
    fd.events = POLLIN;
    fd.revents = 0;
    const int ret = poll(&fd, 1, 100);
    return ret > 0 && (fd.revents & POLLIN);
}

/* "<number> <unit>" with units b, kb, mb, gb (decimal) (:2685-2716) */
size_t parse_bytes(const char *value)
{
    std::istringstream iss(value);
    double base = 0;
    std::string unit;
    iss >> base;
    if (!iss) {
        fprintf(stderr, "could not parse memory value\n");
        return 0;
    }
    iss >> unit;
    if (!iss || unit.empty()) {
        fprintf(stderr, "could not parse memory unit, default to bytes\n");
        unit = "b";
    }
    std::transform(unit.begin(), unit.end(), unit.begin(), ::tolower);
    double mult;
    if (unit == "b" || unit == "byte" || unit == "bytes") mult = 1;
    else if (unit == "kb" || unit == "kbyte" || unit == "kbytes" || unit == "kilobyte" || unit == "kilobytes") mult = 1e3;
    else if (unit == "mb" || unit == "mbyte" || unit == "mbytes" || unit == "megabyte" || unit == "megabytes") mult = 1e6;
    else if (unit == "gb" || unit == "gbyte" || unit == "gbytes" || unit == "gigabyte" || unit == "gigabytes") mult = 1e9;
    else {
        fprintf(stderr, "could not parse byte unit\n");
        return 0;
    }
    return (size_t)(mult * base);
}

struct Text {
    std::vector<unsigned char> T;     /* the packed text, NUL-terminated */
    long n = 0;                        /* characters up to the last sentinel */
    long t = 0;                        /* characters of the database file */
    char sentinel = 0;
    std::vector<long> BEG, END;
    long sid = 0, crossover = -1;
};

/* per pair record, as the batch functions write it */
struct Rec {
    int score, end_query, end_ref, flag, matches, similar, length, pad;
};
static_assert(sizeof(Rec) == sizeof(parasail_b200_record_t), "record layout");

struct Ctx {
    bool is_stats = true, is_trace = false, edge_output = false, graph_output = false;
    bool use_emboss = false, use_ssw = false, use_sam = false, use_sam_header = false;
    bool has_query = false, case_sensitive = false;
    const char *aliases = nullptr;
    int AOL = 80, SIM = 40, OS = 30;
    const parasail_matrix_t *matrix = nullptr;
    Text *text = nullptr;
    parasail_sequences_t *sequences = nullptr, *queries = nullptr;
    FILE *fop = nullptr;
    std::vector<std::vector<std::pair<int, float>>> graph;
    unsigned long edge_count = 0;
};

int self_score(const unsigned char *seq, long len, const parasail_matrix_t *m)
{
    int s = 0;
    for (long i = 0; i < len; ++i) {
        const int c = m->mapper[seq[i]];
        s += m->matrix[m->size * c + c];
    }
    return s;
}

bool saturated(const Ctx &c, int i, int j, int flag, bool with_names)
{
    if (!(flag & PARASAIL_FLAG_SATURATED)) return false;
    if (with_names) {
        if (c.has_query)
            fprintf(stderr, "query %d (%s) and ref %d (%s) saturated\n", i, c.queries->seqs[i].name.s, j,
                    c.sequences->seqs[j].name.s);
        else
            fprintf(stderr, "seq %d (%s) and seq %d (%s) saturated\n", i, c.sequences->seqs[i].name.s, j,
                    c.sequences->seqs[j].name.s);
    } else if (c.has_query) {
        fprintf(stderr, "query %d and ref %d saturated\n", i, j);
    } else {
        fprintf(stderr, "seq %d and seq %d saturated\n", i, j);
    }
    return true;
}

/* score, statistics, edge and graph outputs of one batch
 * (apps/parasail_aligner.cpp:1950-2207) */
void write_records(Ctx &c, const std::vector<Pair> &pairs, const std::vector<Rec> &recs, long start, long stop)
{
    Text &tx = *c.text;
    unsigned long edges = 0;
    for (long k = start; k < stop; ++k) {
        const Rec &r = recs[k - start];
        int i = pairs[k].first, j = pairs[k].second;
        const long i_beg = tx.BEG[i], i_len = tx.END[i] - i_beg;
        const long j_beg = tx.BEG[j], j_len = tx.END[j] - j_beg;
        const int gi = i, gj = j;
        if (c.has_query && !c.graph_output) i -= (int)tx.crossover;
        if (saturated(c, c.graph_output ? gi : i, j, r.flag, false)) continue;
        if (c.is_stats && (c.edge_output || c.graph_output)) {
            const int iss = self_score(&tx.T[i_beg], i_len, c.matrix);
            const int jss = self_score(&tx.T[j_beg], j_len, c.matrix);
            long max_len;
            int ss;
            if (i_len > j_len) { max_len = i_len; ss = iss; }
            else { max_len = j_len; ss = jss; }
            if ((long)r.length * 100 >= (long)c.AOL * (int)max_len && r.matches * 100 >= c.SIM * r.length &&
                r.score * 100 >= c.OS * ss) {
                if (c.edge_output) {
                    ++edges;
                    fprintf(c.fop, "%d,%d,%f,%f,%f\n", i, j, 1.0 * r.length / max_len, 1.0 * r.matches / r.length,
                            1.0 * r.score / ss);
                } else {
                    const float v = (float)(1.0 * r.length / max_len);
                    ++c.edge_count;
                    c.graph[gi].push_back(std::make_pair(gj, v));
                    c.graph[gj].push_back(std::make_pair(gi, v));
                }
            }
        } else if (c.is_stats) {
            fprintf(c.fop, "%d,%d,%ld,%ld,%d,%d,%d,%d,%d,%d\n", i, j, i_len, j_len, r.score, r.end_query,
                    r.end_ref, r.matches, r.similar, r.length);
        } else {
            fprintf(c.fop, "%d,%d,%ld,%ld,%d,%d,%d\n", i, j, i_len, j_len, r.score, r.end_query, r.end_ref);
        }
    }
    if (c.edge_output) fprintf(stdout, "%20s: %lu\n", "edges count", edges);
}

/* EMBOSS, SSW and SAM outputs of a batch of trace results
 * (apps/parasail_aligner.cpp:2210-2517) */
void write_traces(Ctx &c, const std::vector<Pair> &pairs, const std::vector<parasail_result_t *> &res, long start,
                  long stop)
{
    if (c.use_sam && c.use_sam_header && c.has_query && start == 0) {
        fprintf(c.fop, "@HD\tVN:1.4\tSO:queryname\n");
        for (size_t k = 0; k < c.sequences->l; ++k)
            fprintf(c.fop, "@SQ\tSN:%s\tLN:%d\n", c.sequences->seqs[k].name.s, (int32_t)c.sequences->seqs[k].seq.l);
    }
    for (long k = start; k < stop; ++k) {
        parasail_result_t *r = res[k - start];
        int i = pairs[k].first;
        const int j = pairs[k].second;
        if (c.has_query) i -= (int)c.text->crossover;
        if (!r) continue;
        if (saturated(c, i, j, r->flag, true)) continue;
        const parasail_sequence_t &ref_seq = c.sequences->seqs[j];
        const parasail_sequence_t &read_seq = c.has_query ? c.queries->seqs[i] : c.sequences->seqs[i];
        if (c.use_emboss) {
            parasail_traceback_generic_extra2(read_seq.seq.s, (int)read_seq.seq.l, ref_seq.seq.s, (int)ref_seq.seq.l,
                                              read_seq.name.s, ref_seq.name.s, c.matrix, r, '|', ':', '.', 50, 14, 1,
                                              7, c.fop, c.case_sensitive, c.aliases);
        } else if (c.use_ssw) {
            fprintf(c.fop, "target_name: %s\n", ref_seq.name.s);
            fprintf(c.fop, "query_name: %s\n", read_seq.name.s);
            parasail_cigar_t *cg = parasail_result_get_cigar_extra(r, read_seq.seq.s, (int)read_seq.seq.l,
                                                                   ref_seq.seq.s, (int)ref_seq.seq.l, c.matrix,
                                                                   c.case_sensitive, c.aliases);
            fprintf(c.fop,
                    "optimal_alignment_score: %d\tstrand: +\ttarget_begin: %d\ttarget_end: %d\tquery_begin: %d"
                    "\tquery_end: %d\n",
                    r->score, cg->beg_ref + 1, parasail_result_get_end_ref(r) + 1, cg->beg_query + 1,
                    parasail_result_get_end_query(r) + 1);
            parasail_cigar_free(cg);
            parasail_traceback_generic_extra2(read_seq.seq.s, (int)read_seq.seq.l, ref_seq.seq.s, (int)ref_seq.seq.l,
                                              "Query:", "Target:", c.matrix, r, '|', '*', '*', 60, 10, 0, 7, c.fop,
                                              c.case_sensitive, c.aliases);
        } else {
            fprintf(c.fop, "%s\t", read_seq.name.s);
            if (r->score == 0) {
                fprintf(c.fop, "4\t*\t0\t255\t*\t*\t0\t0\t*\t*\n");
                continue;
            }
            parasail_cigar_t *cg = parasail_result_get_cigar_extra(r, read_seq.seq.s, (int)read_seq.seq.l,
                                                                   ref_seq.seq.s, (int)ref_seq.seq.l, c.matrix,
                                                                   c.case_sensitive, c.aliases);
            uint32_t mismatch = 0;
            fprintf(c.fop, "0\t");
            fprintf(c.fop, "%s\t%d\t%d\t", ref_seq.name.s, cg->beg_ref + 1, 255);
            if (parasail_result_is_sw(r) && cg->beg_query > 0) fprintf(c.fop, "%dS", cg->beg_query);
            for (int e = 0; e < cg->len; ++e) {
                const char op = parasail_cigar_decode_op(cg->seq[e]);
                const uint32_t len = parasail_cigar_decode_len(cg->seq[e]);
                fprintf(c.fop, "%lu%c", (unsigned long)len, op);
                if (op == 'X' || op == 'I' || op == 'D') mismatch += len;
            }
            const int32_t tail = (int32_t)read_seq.seq.l - r->end_query - 1;
            if (parasail_result_is_sw(r) && tail > 0) fprintf(c.fop, "%dS", tail);
            fprintf(c.fop, "\t*\t0\t0\t");
            fprintf(c.fop, "%s", read_seq.seq.s);
            fprintf(c.fop, "\t");
            if (read_seq.qual.s) fprintf(c.fop, "%s", read_seq.qual.s);
            else fprintf(c.fop, "*");
            fprintf(c.fop, "\tAS:i:%d", r->score);
            fprintf(c.fop, "\tNM:i:%d\t", mismatch);
            fprintf(c.fop, "\n");
            parasail_cigar_free(cg);
        }
    }
}

/* batch boundaries (apps/parasail_aligner.cpp:414-573): a fixed size, else
 * the trace tables' bytes (one per cell) or the results that fit the budget */
std::vector<long> calc_batches(long long batch_size, size_t budget, bool is_trace, bool is_stats,
                               const std::vector<Pair> &pairs, const Text &tx)
{
    std::vector<long> b;
    b.push_back(0);
    const size_t np = pairs.size();
    if (batch_size != 0) {
        for (size_t k = (size_t)batch_size; k < np; k += (size_t)batch_size) b.push_back((long)k);
        b.push_back((long)np);
        return b;
    }
    if (is_trace) {
        size_t cur = 0;
        for (size_t k = 0; k < np; ++k) {
            const size_t local = (size_t)(tx.END[pairs[k].first] - tx.BEG[pairs[k].first]) *
                                 (size_t)(tx.END[pairs[k].second] - tx.BEG[pairs[k].second]);
            if (k > 0 && cur + local > budget) {
                b.push_back((long)k);
                cur = local;
            } else {
                cur += local;
            }
        }
        b.push_back((long)np);
        return b;
    }
    size_t rsize = sizeof(parasail_result_t) + (is_stats ? sizeof(parasail_result_extra_stats_t) : 0);
    size_t per = budget / rsize;
    if (per == 0) per = 1;
    for (size_t k = 1; k <= np / per; ++k) b.push_back((long)(k * per));
    if (b.back() != (long)np) b.push_back((long)np);
    return b;
}

}  // namespace

int main(int argc, char **argv)
{
    const char *fname = nullptr, *qname = nullptr, *oname = "parasail.csv";
    bool oname_from_user = false, use_filter = true, use_dna = false, pairs_only = false, verbose = false;
    bool verbose_memory = false;
    const char *funcname = "sw_stats_striped_16", *matrixname = nullptr, *output_format = nullptr;
    int cutoff = 7, gap_open = 10, gap_extend = 1, match = 1, mismatch = 0, kbandsize = 3;
    long long batch_size = 0;
    size_t memory_budget = (size_t)4 << 30;
    bool matrix_needs_free = false;
    Ctx c;
    int opt;
    while ((opt = getopt(argc, argv, "a:A:b:c:Cde:Ef:g:Ghi:k:l:m:M:o:O:pq:r:s:t:vVxX:")) != -1) {
        switch (opt) {
            case 'a': funcname = optarg; break;
            case 'A': c.aliases = optarg; break;
            case 'b': {
                std::istringstream iss(optarg);
                iss >> batch_size;
                if (batch_size < 0) {
                    fprintf(stderr, "batch size must be >= 0\n");
                    print_help(EXIT_FAILURE);
                }
                break;
            }
            case 'c':
                cutoff = atoi(optarg);
                if (cutoff <= 0) {
                    fprintf(stderr, "cutoff must be > 0\n");
                    print_help(EXIT_FAILURE);
                }
                break;
            case 'C': c.case_sensitive = true; break;
            case 'd': use_dna = true; break;
            case 'e':
                gap_extend = atoi(optarg);
                if (gap_extend < 0) {
                    fprintf(stderr, "gap extend must be >= 0\n");
                    print_help(EXIT_FAILURE);
                }
                break;
            case 'E': c.edge_output = true; break;
            case 'f': fname = optarg; break;
            case 'g': oname = optarg; oname_from_user = true; break;
            case 'G': c.graph_output = true; break;
            case 'h': print_help(EXIT_FAILURE); break;
            case 'i': c.OS = atoi(optarg); if (c.OS < 0 || c.OS > 100) print_help(EXIT_FAILURE); break;
            case 'k':
                kbandsize = atoi(optarg);
                if (kbandsize <= 0) {
                    fprintf(stderr, "band size must be > 0\n");
                    print_help(EXIT_FAILURE);
                }
                break;
            case 'l': c.AOL = atoi(optarg); if (c.AOL < 0 || c.AOL > 100) print_help(EXIT_FAILURE); break;
            case 'm': matrixname = optarg; break;
            case 'M': match = atoi(optarg); if (match < 0) print_help(EXIT_FAILURE); break;
            case 'o':
                gap_open = atoi(optarg);
                if (gap_open < 0) {
                    fprintf(stderr, "gap open must be >= 0\n");
                    print_help(EXIT_FAILURE);
                }
                break;
            case 'O': output_format = optarg; break;
            case 'p': pairs_only = true; break;
            case 'q': qname = optarg; break;
            case 'r': memory_budget = parse_bytes(optarg); break;
            case 's': c.SIM = atoi(optarg); if (c.SIM < 0 || c.SIM > 100) print_help(EXIT_FAILURE); break;
            case 't': break;
            case 'v': verbose = true; break;
            case 'V': verbose_memory = true; break;
            case 'x': use_filter = false; break;
            case 'X': mismatch = atoi(optarg); if (mismatch < 0) print_help(EXIT_FAILURE); break;
            default: print_help(EXIT_FAILURE);
        }
    }
    /* the function */
    bool is_banded = false;
    if (strstr(funcname, "profile")) {
        if (!parasail_lookup_pfunction_info(funcname)) {
            fprintf(stderr, "Specified profile function not found.\n");
            exit(EXIT_FAILURE);
        }
    } else if (!parasail_lookup_function_info(funcname)) {
        if (strstr(funcname, "nw_banded")) {
            is_banded = true;
        } else {
            fprintf(stderr, "Specified function not found.\n");
            exit(EXIT_FAILURE);
        }
    }
    /* inputs: a file and an optional query file, or standard input */
    if (stdin_has_data()) {
        if (!fname) fname = "stdin";
        else if (!qname) { qname = "stdin"; c.has_query = true; }
        else {
            fprintf(stderr, "input file, query file, and stdin detected; max inputs is 2\n");
            exit(EXIT_FAILURE);
        }
    } else if (!fname) {
        fprintf(stderr, "missing input file\n");
        print_help(EXIT_FAILURE);
    } else if (qname) {
        c.has_query = true;
    }
    c.is_trace = strstr(funcname, "trace") != nullptr;
    c.is_stats = strstr(funcname, "stats") != nullptr;
    if (c.edge_output && c.graph_output) {
        fprintf(stderr, "Can only request one of edge or graph output.\n");
        exit(EXIT_FAILURE);
    }
    if ((c.edge_output || c.graph_output) && !c.is_stats) {
        fprintf(stderr, "Edge or graph output requested, but alignment function does not return statistics.\n");
        exit(EXIT_FAILURE);
    }
    if (c.graph_output && c.has_query) {
        fprintf(stderr, "Cannot specify a query file and output as a graph.\n");
        exit(EXIT_FAILURE);
    }
    if (output_format) {
        bool trace_warning = true;
        if (strstr(output_format, "SAMH")) { c.use_sam = c.use_sam_header = true; }
        else if (strstr(output_format, "SAM")) { c.use_sam = true; }
        else if (strstr(output_format, "EMBOSS")) { c.use_emboss = true; }
        else if (strstr(output_format, "SSW")) { c.use_ssw = true; }
        else {
            fprintf(stderr, "Unknown output format '%s'.\n", output_format);
            exit(EXIT_FAILURE);
        }
        if (!c.is_trace && trace_warning) {
            fprintf(stderr, "The selected output format '%s' requires an alignment function that returns a traceback.\n",
                    output_format);
            exit(EXIT_FAILURE);
        }
    } else if (c.is_trace) {
        fprintf(stderr, "Please select trace output format.\n");
        exit(EXIT_FAILURE);
    }
    /* the substitution matrix */
    if (!matrixname && use_dna) {
        matrixname = "ACGT";
        c.matrix = c.case_sensitive ? parasail_matrix_create_case_sensitive("ACGT", match, -mismatch)
                                    : parasail_matrix_create("ACGT", match, -mismatch);
        if (!c.matrix) {
            fprintf(stderr, "Could not create DNA match/mismatch matrix.\n");
            exit(EXIT_FAILURE);
        }
        matrix_needs_free = true;
    } else {
        if (!matrixname) matrixname = "blosum62";
        c.matrix = parasail_matrix_lookup(matrixname);
        if (!c.matrix) {
            c.matrix = c.case_sensitive ? parasail_matrix_from_file_case_sensitive(matrixname)
                                        : parasail_matrix_from_file(matrixname);
            if (!c.matrix) {
                fprintf(stderr, "parasail_matrix_from_file(%s) failed.\n", matrixname);
                exit(EXIT_FAILURE);
            }
            matrix_needs_free = true;
        }
    }
    if (c.matrix->type == PARASAIL_MATRIX_TYPE_PSSM) {
        fprintf(stderr, "PSSM matrices are not supported by %s (the batch kernels take square matrices).\n",
                g_progname);
        exit(EXIT_FAILURE);
    }
    if (c.is_trace && !oname_from_user) oname = "stdout";
    if (verbose) {
        fprintf(stdout,
                "%20s: %s\n%20s: %d\n%20s: %s\n%20s: %s\n%20s: %s\n%20s: %d\n%20s: %d\n%20s: %s\n%20s: %d\n"
                "%20s: %d\n%20s: %d\n%20s: %s\n%20s: %s\n%20s: %s\n%20s: %lld\n%20s: %.4f GB\n",
                "funcname", funcname, "cutoff", cutoff, "case sensitive", c.case_sensitive ? "yes" : "no",
                "alphabet aliases", c.aliases ? c.aliases : "<no aliases>", "use filter", use_filter ? "yes" : "no",
                "gap_extend", gap_extend, "gap_open", gap_open, "matrix", matrixname, "AOL", c.AOL, "SIM", c.SIM,
                "OS", c.OS, "file", fname, "query", qname ? qname : "<no query>", "output", oname, "batch_size",
                batch_size, "memory_budget", memory_budget * 1e-9);
        if (use_dna) fprintf(stdout, "%20s: %d\n%20s: %d\n", "match", match, "mismatch", mismatch);
    }
    if (oname_from_user || !c.is_trace) {
        if (!(c.fop = fopen(oname, "w"))) {
            fprintf(stderr, "%s: Cannot open output file `%s': ", g_progname, oname);
            perror("fopen");
            exit(EXIT_FAILURE);
        }
    } else {
        c.fop = stdout;
    }
    /* the text: database sequences, then query sequences, each followed by
     * '$' (apps/parasail_aligner.cpp:1077-1178) */
    double t0 = now();
    Text tx;
    c.text = &tx;
    {
        size_t count = 0;
        c.sequences = parasail_sequences_from_file(fname);
        if (!c.sequences) {
            fprintf(stderr, "parasail_sequences_from_file(%s) failed.\n", fname);
            exit(EXIT_FAILURE);
        }
        char *T = parasail_sequences_pack(c.sequences, &count);
        if (!T) {
            fprintf(stderr, "parasail_sequences_pack failed.\n");
            exit(EXIT_FAILURE);
        }
        tx.T.assign(T, T + count);
        tx.t = (long)count;
        free(T);
        if (c.has_query) {
            c.queries = parasail_sequences_from_file(qname);
            if (!c.queries) {
                fprintf(stderr, "parasail_sequences_from_file(%s) failed.\n", qname);
                exit(EXIT_FAILURE);
            }
            char *Q = parasail_sequences_pack(c.queries, &count);
            if (!Q) {
                fprintf(stderr, "parasail_sequences_pack queries failed.\n");
                exit(EXIT_FAILURE);
            }
            tx.T.insert(tx.T.end(), Q, Q + count);
            free(Q);
        }
        tx.T.push_back('\0');
    }
    long n = (long)tx.T.size() - 1;
    if (verbose) fprintf(stdout, "%20s: %.4f seconds\n", "read and pack time", now() - t0);
    /* the sentinel is the last printable character; the text ends there */
    {
        long off = 0;
        while (n - off > 0 && !isgraph(tx.T[n - off])) ++off;
        tx.sentinel = (char)tx.T[n - off];
        n = n - off + 1;
    }
    for (long i = 0; i < n; ++i) tx.sid += tx.T[i] == (unsigned char)tx.sentinel;
    if (tx.sid == 0) {
        fprintf(stderr, "no sentinal(%c) found in input\n", tx.sentinel);
        exit(EXIT_FAILURE);
    }
    tx.BEG.push_back(0);
    {
        bool lower = false, upper = false;
        for (long i = 0; i < n; ++i) {
            if (tx.T[i] == (unsigned char)tx.sentinel) {
                tx.END.push_back(i);
                tx.BEG.push_back(i + 1);
                if (tx.crossover == -1 && i >= tx.t) tx.crossover = (long)tx.END.size() - 1;
            }
            lower = lower || (tx.T[i] >= 'a' && tx.T[i] <= 'z');
            upper = upper || (tx.T[i] >= 'A' && tx.T[i] <= 'Z');
        }
        /* the filter compares upper-cased text when both cases occur */
        if (use_filter && lower && upper && !c.case_sensitive)
            for (long i = 0; i < n; ++i) tx.T[i] = (unsigned char)toupper(tx.T[i]);
    }
    if (!c.has_query) tx.crossover = -1;
    const int nseq = (int)tx.sid;
    /* the pairs */
    std::vector<Pair> pairs;
    t0 = now();
    if (use_filter) {
        int *pp = nullptr;
        size_t np = 0;
        if (parasail_b200_candidate_pairs((const char *)tx.T.data(), (size_t)n, tx.sentinel, cutoff,
                                          c.has_query ? tx.t : -1, &pp, &np) != 0) {
            fprintf(stderr, "%s: the candidate-pair filter failed.\n", g_progname);
            exit(EXIT_FAILURE);
        }
        pairs.reserve(np);
        for (size_t k = 0; k < np; ++k) pairs.push_back(Pair(pp[2 * k], pp[2 * k + 1]));
        free(pp);
        if (verbose) {
            fprintf(stdout, "%20s: %.4f seconds\n", "filter time", now() - t0);
            fprintf(stdout, "%20s: %zu\n", "unique pairs", pairs.size());
        }
    } else if (!c.has_query) {
        pairs.reserve((size_t)nseq * (nseq > 0 ? nseq - 1 : 0) / 2);
        for (int i = 0; i < nseq; ++i)
            for (int j = i + 1; j < nseq; ++j) pairs.push_back(Pair(i, j));
    } else {
        for (int i = (int)tx.crossover; i < nseq; ++i)
            for (int j = 0; j < (int)tx.crossover; ++j) pairs.push_back(Pair(i, j));
    }
    if (!c.is_trace && pairs_only) {
        if (pairs.empty()) {
            fprintf(stderr, "pairs and vpairs were empty\n");
            exit(EXIT_FAILURE);
        }
        for (const Pair &p : pairs) fprintf(c.fop, "%d,%d\n", p.first, p.second);
        fclose(c.fop);
        return 0;
    }
    if (pairs.empty()) {
        if (use_filter)
            fprintf(stderr, "no alignment work, either the filter removed all alignments or the input file(s) were empty\n");
        else
            fprintf(stderr, "no alignment work, perhaps the input file(s) were empty\n");
        exit(EXIT_FAILURE);
    }
    if (c.graph_output) c.graph.resize((size_t)nseq);
    /* alignment in batches; a batch's output is written while the next aligns */
    t0 = now();
    const std::vector<long> batches = calc_batches(batch_size, memory_budget, c.is_trace, c.is_stats, pairs, tx);
    if (verbose_memory)
        for (size_t b = 0; b + 1 < batches.size(); ++b)
            fprintf(stdout, "%20s: %ld-%ld\n", "batch", batches[b], batches[b + 1]);
    parasail_b200_seqdb_t *db = nullptr;
    if (!c.is_trace && !is_banded) {
        db = parasail_b200_seqdb_create((const char *)tx.T.data(), (size_t)n, tx.sentinel, c.matrix);
        if (!db) {
            fprintf(stderr, "%s: cannot place the sequences on the device.\n", g_progname);
            exit(EXIT_FAILURE);
        }
    }
    std::vector<int64_t> offs((size_t)nseq);
    std::vector<int> lens((size_t)nseq);
    for (int s = 0; s < nseq; ++s) {
        offs[(size_t)s] = tx.BEG[(size_t)s];
        lens[(size_t)s] = (int)(tx.END[(size_t)s] - tx.BEG[(size_t)s]);
    }
    std::thread writer;
    std::vector<Rec> recs[2];
    std::vector<parasail_result_t *> traces[2];
    unsigned long long work = 0;
    for (size_t b = 0; b + 1 < batches.size(); ++b) {
        const long start = batches[b], stop = batches[b + 1];
        const int nb = (int)(stop - start);
        const int slot = (int)(b & 1);
        std::vector<int> first((size_t)nb), second((size_t)nb);
        for (int k = 0; k < nb; ++k) {
            first[(size_t)k] = pairs[(size_t)(start + k)].first;
            second[(size_t)k] = pairs[(size_t)(start + k)].second;
            work += (unsigned long long)lens[(size_t)first[(size_t)k]] * (unsigned long long)lens[(size_t)second[(size_t)k]];
        }
        int rc = 0;
        if (c.is_trace) {
            std::vector<int64_t> qo((size_t)nb), to((size_t)nb);
            std::vector<int> ql((size_t)nb), tl((size_t)nb);
            for (int k = 0; k < nb; ++k) {
                qo[(size_t)k] = offs[(size_t)first[(size_t)k]];
                ql[(size_t)k] = lens[(size_t)first[(size_t)k]];
                to[(size_t)k] = offs[(size_t)second[(size_t)k]];
                tl[(size_t)k] = lens[(size_t)second[(size_t)k]];
            }
            traces[slot].assign((size_t)nb, nullptr);
            rc = parasail_b200_batch_pairs_trace(funcname, c.matrix, (const char *)tx.T.data(), qo.data(), ql.data(),
                                                 (const char *)tx.T.data(), to.data(), tl.data(), nb, gap_open,
                                                 gap_extend, traces[slot].data());
        } else if (is_banded) {
            std::vector<int64_t> qo((size_t)nb), to((size_t)nb);
            std::vector<int> ql((size_t)nb), tl((size_t)nb), sc((size_t)nb);
            for (int k = 0; k < nb; ++k) {
                qo[(size_t)k] = offs[(size_t)first[(size_t)k]];
                ql[(size_t)k] = lens[(size_t)first[(size_t)k]];
                to[(size_t)k] = offs[(size_t)second[(size_t)k]];
                tl[(size_t)k] = lens[(size_t)second[(size_t)k]];
            }
            rc = parasail_b200_nw_banded_batch(c.matrix, (const char *)tx.T.data(), qo.data(), ql.data(),
                                               (const char *)tx.T.data(), to.data(), tl.data(), nb, gap_open,
                                               gap_extend, kbandsize, sc.data());
            recs[slot].assign((size_t)nb, Rec());
            for (int k = 0; k < nb; ++k) {
                Rec &r = recs[slot][(size_t)k];
                r.score = sc[(size_t)k];
                r.end_query = ql[(size_t)k] - 1;
                r.end_ref = tl[(size_t)k] - 1;
                r.flag = PARASAIL_FLAG_NW | PARASAIL_FLAG_BANDED;
            }
        } else {
            recs[slot].assign((size_t)nb, Rec());
            rc = parasail_b200_batch_pairs_seqdb(funcname, c.matrix, db, first.data(), second.data(), (size_t)nb,
                                                 gap_open, gap_extend, memory_budget,
                                                 (parasail_b200_record_t *)recs[slot].data());
        }
        if (writer.joinable()) writer.join();
        if (rc != 0) {
            fprintf(stderr, "%s: alignment of pairs %ld-%ld failed.\n", g_progname, start, stop);
            exit(EXIT_FAILURE);
        }
        if (c.is_trace) {
            writer = std::thread([&c, &pairs, &traces, slot, start, stop]() {
                write_traces(c, pairs, traces[slot], start, stop);
                for (parasail_result_t *r : traces[slot])
                    if (r) parasail_result_free(r);
            });
        } else {
            writer = std::thread([&c, &pairs, &recs, slot, start, stop]() {
                write_records(c, pairs, recs[slot], start, stop);
            });
        }
    }
    if (writer.joinable()) writer.join();
    if (c.graph_output) {
        fprintf(c.fop, "%lu %lu 1\n", (unsigned long)c.graph.size(), c.edge_count);
        for (size_t i = 0; i < c.graph.size(); ++i) {
            if (!c.graph[i].empty()) {
                fprintf(c.fop, "%d %f", c.graph[i][0].first + 1, c.graph[i][0].second);
                for (size_t j = 1; j < c.graph[i].size(); ++j)
                    fprintf(c.fop, "  %d %f", c.graph[i][j].first + 1, c.graph[i][j].second);
                fprintf(c.fop, "\n");
            } else {
                fprintf(c.fop, "\n");
            }
        }
        fprintf(stdout, "%20s: %lu\n", "edges count", c.edge_count);
    }
    const double secs = now() - t0;
    if (verbose) {
        fprintf(stdout, "%20s: %.4f seconds\n", "alignment time", secs);
        fprintf(stdout, "%20s: %llu\n", "work", work);
        fprintf(stdout, "%20s: %.4f\n", "gcups", secs > 0 ? work / secs * 1e-9 : 0.0);
    }
    if (db) parasail_b200_seqdb_free(db);
    if (c.fop != stdout) fclose(c.fop);
    if (c.sequences) parasail_sequences_free(c.sequences);
    if (c.queries) parasail_sequences_free(c.queries);
    if (matrix_needs_free) parasail_matrix_free((parasail_matrix_t *)c.matrix);
    return 0;
}
