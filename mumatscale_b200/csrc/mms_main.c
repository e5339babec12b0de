/*
 * mms_main.c — command-line driver with the reference's interface
 * (ca_main.c:45-53, 120-139):  mmsb200 [-i] -c <deck> [-r <n>]
 *
 * Reads the deck, builds the device-resident domain, runs the reference
 * time loop (loop.c) and prints the same screen lines and grain summary the
 * reference's regression scripts parse (tests/testOneGrain.py,
 * tests/testMultiGrains.py, tests/testAMtrack.py), so those scripts accept
 * this binary in place of muMatScale.  -r <n> restarts from the checkpoint
 * the run loop wrote in the working directory (cp_main.mms, every
 * DataWriteStart steps as the reference's parser sets checkpointfreq); like
 * the reference without DEBUG_CHECKPOINT, n only switches restarting on
 * (ca_main.c:136-137, checkpoint.c:867-960).  Extra options of this build:
 *   -p f32      run the FP32 form instead of the FP64 plain form
 *   -d <n>      CUDA device ordinal
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <unistd.h>

#include "../../include/mms.h"

static void usage(const char *prog)
{
    fprintf(stderr, "Usage: %s [-i] -c <control file> [-r <n>] [-p f64|f32] [-d device]\n", prog);
}

int main(int argc, char **argv)
{
    int interactive = 0, flag, device = 0, prec = MMS_PREC_F64, restart = 0;
    const char *deck = NULL;
    while ((flag = getopt(argc, argv, "ic:r:p:d:h")) != -1) {
        switch (flag) {
        case 'i': interactive = 1; break;
        case 'c': deck = optarg; break;
        case 'r': restart = 1; break;  /* the number is not used (ca_main.c:136-137) */
        case 'p': prec = (strcmp(optarg, "f32") == 0) ? MMS_PREC_F32 : MMS_PREC_F64; break;
        case 'd': device = atoi(optarg); break;
        default: usage(argv[0]); return 1;
        }
    }
    if (!deck) {
        fprintf(stderr, "No Control or Restart file specified.\n");
        usage(argv[0]);
        return 1;
    }
    printf("Start the program... \n");
    mms_params p;
    mms_params_default(&p);
    mms_status st = mms_deck_read(deck, &p);
    if (st != MMS_OK) {
        fprintf(stderr, "error: %s\n", mms_status_string(st));
        return 1;
    }
    p.precision = prec;
    p.device = device;
    printf("Global Configuration:\n");
    printf("Dimensions (Cells):  %d, %d, %d\n", p.gnsbx * p.gsdimx, p.gnsby * p.gsdimy, p.gnsbz * p.gsdimz);
    printf("Num Subblocks:  %d, %d, %d\n", p.gnsbx, p.gnsby, p.gnsbz);
    printf("Form: %s\n", prec == MMS_PREC_F32 ? "FP32" : "FP64 plain");
    struct timeval tv;
    gettimeofday(&tv, NULL);
    double t0 = tv.tv_sec + tv.tv_usec * 1e-6;
    mms_ctx *ctx = NULL;
    st = mms_create(&p, &ctx);
    mms_params_free_lists(&p);
    if (st != MMS_OK) {
        fprintf(stderr, "error: mms_create: %s\n", mms_status_string(st));
        return 1;
    }
    if (restart) {
        st = mms_checkpoint_load(ctx, MMS_CHECKPOINT_FILE);
        if (st != MMS_OK) {
            fprintf(stderr, "error: restart from %s: %s (%s)\n", MMS_CHECKPOINT_FILE, mms_status_string(st),
                    mms_last_error(ctx));
            mms_destroy(ctx);
            return 1;
        }
        uint64_t t = 0;
        mms_get_timestep(ctx, &t);
        printf("task 0 done restarting at timestep %lu\n", (unsigned long)t);
    }
    printf("Initial Subblocks assigned.  Starting calculations.\n");
    st = mms_run(ctx, interactive ? 2 : 1);
    if (st != MMS_OK) {
        fprintf(stderr, "error: %s (%s)\n", mms_status_string(st), mms_last_error(ctx));
        mms_destroy(ctx);
        return 1;
    }
    uint64_t ts = 0;
    mms_get_timestep(ctx, &ts);
    gettimeofday(&tv, NULL);
    printf("Elapsed time:  %lu iterations, %lg sec\n", (unsigned long)ts, tv.tv_sec + tv.tv_usec * 1e-6 - t0);
    mms_destroy(ctx);
    return 0;
}
