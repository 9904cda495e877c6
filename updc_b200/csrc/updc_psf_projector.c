/* Drop-in replacement for the reference PSF projector executable
 * (updc/c_core/psf_projector.c:245-268): "manifest workers results.csv",
 * --self-test, the projected PSF files, the results CSV and the
 * "UPDC_PSF_PROJECT: <msg>" failures with exit status 1; each projection runs
 * on the GPU through libupdc_b200.so (the workers argument is accepted: the
 * GPU handles one job at a time). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/updc_b200.h"

typedef struct {
    char input[1024], vertices[1024], output[1024];
    int width, height, out_width, out_height;
    double input_sum, output_sum, rel;
    uint64_t overlaps;
} Job;

static void die(const char *message) {
    fprintf(stderr, "UPDC_PSF_PROJECT: %s\n", message);
    exit(EXIT_FAILURE);
}

/* The manifest format (updc/_engine.py writes it, psf_projector.c reads it):
 * one job per line, tab-separated "input width height vertices output label",
 * empty lines and lines starting with '#' ignored; runs of separators count
 * as one and fields after the sixth are ignored.  The file is read whole,
 * the lines are counted to size the job array once, then each line is cut
 * into its fields in place. */
static char *read_text(const char *path, size_t *len) {
    FILE *f = fopen(path, "rb");
    if (!f) die("cannot open PSF projection manifest");
    size_t cap = 4096, n = 0;
    char *text = malloc(cap + 1);
    if (!text) die("out of memory");
    for (;;) {
        const size_t got = fread(text + n, 1, cap - n, f);
        n += got;
        if (n < cap) break;
        cap *= 2;
        char *grown = realloc(text, cap + 1);
        if (!grown) die("out of memory");
        text = grown;
    }
    fclose(f);
    text[n] = '\0';
    *len = n;
    return text;
}

static int is_separator(char c) { return c == '\t' || c == '\r'; }

/* Cuts the line at p (NUL-terminated) into at most `want` fields. */
static int split_fields(char *p, char **field, int want) {
    int count = 0;
    while (*p && count < want) {
        while (*p && is_separator(*p)) ++p;
        if (!*p) break;
        field[count++] = p;
        while (*p && !is_separator(*p)) ++p;
        if (*p) *p++ = '\0';
    }
    return count;
}

static int copy_path(char *dst, size_t cap, const char *src) {
    const size_t n = strlen(src);
    if (n >= cap) return 0;
    memcpy(dst, src, n + 1);
    return 1;
}

static Job *parse_jobs(const char *path, int *njobs) {
    size_t len = 0;
    char *text = read_text(path, &len);
    size_t lines = 1;
    for (size_t i = 0; i < len; ++i) lines += text[i] == '\n';
    Job *jobs = calloc(lines, sizeof(Job));
    if (!jobs) die("out of memory");
    int n = 0;
    for (char *line = text; line && *line;) {
        char *next = strchr(line, '\n');
        if (next) *next++ = '\0';
        if (line[0] != '\0' && line[0] != '#') {
            char *field[6];
            if (split_fields(line, field, 6) < 6) die("PSF manifest needs input,width,height,vertices,output,label");
            Job *job = &jobs[n++];
            if (!copy_path(job->input, sizeof(job->input), field[0]) ||
                !copy_path(job->vertices, sizeof(job->vertices), field[3]) ||
                !copy_path(job->output, sizeof(job->output), field[4]))
                die("PSF manifest path too long");
            job->width = (int)strtol(field[1], NULL, 10);
            job->height = (int)strtol(field[2], NULL, 10);
            if (job->width < 1 || job->height < 1) die("invalid PSF input dimensions");
        }
        line = next;
    }
    free(text);
    if (n < 1) die("empty PSF projection manifest");
    *njobs = n;
    return jobs;
}

int main(int argc, char **argv) {
    if (argc == 2 && strcmp(argv[1], "--self-test") == 0) {
        const double quad[8] = {-0.5, -0.5, -0.5, 0.5, 0.5, 0.5, 0.5, -0.5};
        const float a = updc_polygon_area(quad, 4), o = updc_overlap_area(quad, 0, 0);
        if ((a > 1.0f ? a - 1.0f : 1.0f - a) > 2.0e-6f || (o > 1.0f ? o - 1.0f : 1.0f - o) > 2.0e-6f) return 1;
        printf("UPDC PSF projector self-test: OK\n");
        return 0;
    }
    if (argc != 4) die("usage: updc_psf_projector manifest workers results.csv");
    int n = 0;
    Job *jobs = parse_jobs(argv[1], &n);
    for (int i = 0; i < n; ++i) {
        Job *j = &jobs[i];
        char msg[512];
        const int rc = updc_psf_project_file(j->input, j->width, j->height, j->vertices, j->output, &j->out_width,
                                             &j->out_height, &j->input_sum, &j->output_sum, &j->overlaps, msg,
                                             sizeof(msg));
        if (rc == 2) {
            fprintf(stderr, "UPDC_PSF_PROJECT: exposure %d flux mismatch input=%.17g output=%.17g rel=%.6g\n", i + 1,
                    j->input_sum, j->output_sum, (j->output_sum - j->input_sum) / j->input_sum);
            die(msg);
        }
        if (rc) die(msg);
        j->rel = (j->output_sum - j->input_sum) / j->input_sum;
        printf("PSF polygon %d/%d: %dx%d -> %dx%d, overlaps=%llu, flux rel=%.3e\n", i + 1, n, j->width, j->height,
               j->out_width, j->out_height, (unsigned long long)j->overlaps, j->rel);
        fflush(stdout);
    }
    FILE *r = fopen(argv[3], "w");
    if (!r) die("cannot create PSF projection results");
    fprintf(r, "exposure,width,height,input_sum,output_sum,flux_rel_error,overlaps\n");
    for (int i = 0; i < n; ++i) {
        const Job *j = &jobs[i];
        fprintf(r, "%d,%d,%d,%.17g,%.17g,%.17g,%llu\n", i + 1, j->out_width, j->out_height, j->input_sum,
                j->output_sum, j->rel, (unsigned long long)j->overlaps);
    }
    if (fclose(r)) die("cannot close PSF projection results");
    free(jobs);
    return 0;
}
