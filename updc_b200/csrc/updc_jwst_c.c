/* Drop-in replacement for the frozen core executable (updc/c_core/updc_core.c:1566-1572):
 * the same 18 positional arguments, --self-test, outputs and "UPDC_ALL: <msg>" failures,
 * with the solve running on the B200 through libupdc_b200.so. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/updc_b200.h"

int main(int argc, char **argv) {
    if (argc == 2 && strcmp(argv[1], "--self-test") == 0) {
        char msg[256];
        const int rc = updc_self_test(msg, sizeof(msg));
        if (rc) fprintf(stderr, "%s\n", msg);
        else printf("%s\n", msg);
        return rc;
    }
    if (argc != 19) {
        fprintf(stderr, "UPDC_ALL: usage: updc_jwst_c manifest width height input_width input_height exposures "
                        "psf_transposed iterations iter_prefix wht.bin fft_workers exposure_workers preprocess_workers "
                        "plan_measure autotune retune_fft wisdom_path save_every\n");
        return EXIT_FAILURE;
    }
    UPDC_ALL(argv[1], atoi(argv[2]), atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]), atoi(argv[7]),
             atoi(argv[8]), argv[9], argv[10], atoi(argv[11]), atoi(argv[12]), atoi(argv[13]), atoi(argv[14]),
             atoi(argv[15]), atoi(argv[16]), argv[17], atoi(argv[18]));
    return 0;
}
