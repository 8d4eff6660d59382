/*
 * pf_cli.c -- command line of the reference driver (pf_generic_soa.cu:582-684):
 *   pf_cli [-m particles[:max]] [-N subfilters[:max]] [-t transfer[:max]]
 *          [-r resampling_freq] [-l loops] [-d device] [-M arm|unicycle] input_file
 * Prints "N m t e" and one line per run with the mean estimate error.
 * -M unicycle runs the unicycle program's filter and trace format instead
 * (src/models/unicycle/particle_filter.cu:596-650; -r does not apply).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "esthera_b200.h"

static void parse_range(const char* s, int* lo, int* hi)
{
    const char* c = strchr(s, ':');
    *lo = atoi(s);
    *hi = c ? atoi(c + 1) : *lo;
}

int main(int argc, char** argv)
{
    int t0 = 1, t1 = 1, n0 = 16, n1 = 16, m0 = 256, m1 = 256, loops = 1, device = 0, unicycle = 0, opt;
    float freq = 1.0f;
    while ((opt = getopt(argc, argv, "m:N:t:r:l:d:M:")) != -1) {
        switch (opt) {
        case 'm': parse_range(optarg, &m0, &m1); break;
        case 'N': parse_range(optarg, &n0, &n1); break;
        case 't': parse_range(optarg, &t0, &t1); break;
        case 'r': freq = (float)atof(optarg); break;
        case 'l': loops = atoi(optarg); break;
        case 'd': device = atoi(optarg); break;
        case 'M':
            if (strcmp(optarg, "unicycle") == 0) {
                unicycle = 1;
            } else if (strcmp(optarg, "arm") != 0) {
                fprintf(stderr, "unknown model %s (arm, unicycle)\n", optarg);
                return 1;
            }
            break;
        default:
            fprintf(stderr,
                    "Usage: %s [-m #particles] [-N #cores] [-t #transfer] [-r resamplingChance] [-M arm|unicycle] "
                    "input_file\n",
                    argv[0]);
            return 1;
        }
    }
    if (optind >= argc) {
        fprintf(stderr, "no input file given\n");
        return 1;
    }
    (void)device;
    printf("N m t e\n");
    for (int t = t0; t <= t1; ++t)
        for (int n = n0; n <= n1; n *= 2)
            for (int m = m0; m <= m1; m *= 2)
                for (int l = 0; l < loops; ++l) {
                    float e = 0.0f;
                    pf_status s = unicycle ? pf_beacon_particle_filter(m, n, t, argv[optind], &e)
                                           : pf_particle_filter(m, n, t, freq, argv[optind], &e);
                    if (s != PF_OK) {
                        fprintf(stderr, "error: %s (%s)\n", pf_status_string(s), pf_last_error());
                        return 1;
                    }
                    printf("%d %d %d %.16f\n", n, m, t, e);
                }
    return 0;
}
