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

int main(int argc, char **argv) {
    if (argc == 2 && strcmp(argv[1], "--self-test") == 0) {
        const double quad[8] = {-0.5, -0.5, -0.5, 0.5, 0.5, 0.5, 0.5, -0.5};
        const float a = updc_polygon_area(quad, 4), o = updc_overlap_area(quad, 0, 0);
        if ((a > 1.0f ? a - 1.0f : 1.0f - a) > 2.0e-6f || (o > 1.0f ? o - 1.0f : 1.0f - o) > 2.0e-6f) return 1;
        printf("UPDC PSF projector self-test: OK\n");
        return 0;
    }
    if (argc != 4) die("usage: updc_psf_projector manifest workers results.csv");
    FILE *f = fopen(argv[1], "r");
    if (!f) die("cannot open PSF projection manifest");
    int cap = 16, n = 0;
    Job *jobs = calloc((size_t)cap, sizeof(Job));
    char line[8192];
    while (jobs && fgets(line, sizeof(line), f)) {
        if (line[0] == '\0' || line[0] == '\n' || line[0] == '#') continue;
        if (n == cap) {
            cap *= 2;
            Job *t = realloc(jobs, (size_t)cap * sizeof(Job));
            if (!t) die("out of memory expanding jobs");
            jobs = t;
            memset(jobs + n, 0, (size_t)(cap - n) * sizeof(Job));
        }
        char *save = NULL, *field[6];
        for (int j = 0; j < 6; ++j) field[j] = strtok_r(j ? NULL : line, "\t\r\n", &save);
        for (int j = 0; j < 6; ++j)
            if (!field[j]) die("PSF manifest needs input,width,height,vertices,output,label");
        Job *job = &jobs[n++];
        if (strlen(field[0]) >= sizeof(job->input) || strlen(field[3]) >= sizeof(job->vertices) ||
            strlen(field[4]) >= sizeof(job->output))
            die("PSF manifest path too long");
        strcpy(job->input, field[0]);
        job->width = (int)strtol(field[1], NULL, 10);
        job->height = (int)strtol(field[2], NULL, 10);
        strcpy(job->vertices, field[3]);
        strcpy(job->output, field[4]);
        if (job->width < 1 || job->height < 1) die("invalid PSF input dimensions");
    }
    fclose(f);
    if (!jobs) die("out of memory");
    if (n < 1) die("empty PSF projection manifest");
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
