/*
 * pennant_oracle_main.c -- command-line front end of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Mirrors the reference's `pennant -f deck.pnt`
 * (main.cc:46-107, Driver::run Driver.cc:102-187): runs the deck and writes
 * <probname>.xy and the EnSight Gold set next to an output base name.
 *
 *   pennant_oracle [-t threads] -f deck.pnt [-o outbase]
 */
#include "pnt_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

int main(int argc, char** argv) {
    const char* deck = NULL;
    const char* outbase = NULL;
    int threads = 1;
    for (int i = 1; i < argc; ++i) {
        if (!strcmp(argv[i], "-f") && i + 1 < argc) deck = argv[++i];
        else if (!strcmp(argv[i], "-o") && i + 1 < argc) outbase = argv[++i];
        else if (!strcmp(argv[i], "-t") && i + 1 < argc) threads = atoi(argv[++i]);
        else { fprintf(stderr, "Usage: pennant_oracle [-t threads] -f deck.pnt [-o outbase]\n"); return 2; }
    }
    if (!deck) { fprintf(stderr, "No input file specified\n"); return 2; }
    char err[512] = {0};
    orc_sim* sim = NULL;
    int st = orc_create(deck, NULL, &sim, err, sizeof(err));
    if (st) { fprintf(stderr, "Error: %s\n", err); return 1; }
    orc_set_threads(sim, threads);
    printf("--- Mesh Information ---\nPoints:  %lld\nZones:   %lld\nSides:   %lld\n",
           (long long)orc_num(sim, "nump"), (long long)orc_num(sim, "numz"),
           (long long)orc_num(sim, "nums"));
    const int dtreport = (int)orc_num(sim, "dtreport");
    struct timespec t0, t1, tp;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    tp = t0;
    while (!orc_done(sim)) {
        st = orc_cycle(sim);
        if (st) {
            fprintf(stderr, "Error: %lld negative side volumes on cycle %lld\nExiting...\n",
                    (long long)orc_num(sim, "nbad"), (long long)orc_num(sim, "cycle"));
            orc_destroy(sim);
            return 1;
        }
        const int cyc = (int)orc_num(sim, "cycle");
        if (cyc == 1 || cyc % dtreport == 0) {
            clock_gettime(CLOCK_MONOTONIC, &t1);
            long long us = (long long)((t1.tv_sec - tp.tv_sec) * 1000000LL + (t1.tv_nsec - tp.tv_nsec) / 1000);
            tp = t1;
            printf("End cycle %6d, time = %11.5g, dt = %11.5g, wall = %11lld us\n", cyc,
                   orc_scalar(sim, "time"), orc_scalar(sim, "dt"), us);
        }
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    const double wall = (t1.tv_sec - t0.tv_sec) * 1e6 + (t1.tv_nsec - t0.tv_nsec) / 1e3;
    printf("\nRun complete\ncycle = %6lld,        cstop = %8lld\ntime = %14.6g, tstop = %8.6g\n\n",
           (long long)orc_num(sim, "cycle"), (long long)orc_num(sim, "cstop"),
           orc_scalar(sim, "time"), orc_scalar(sim, "tstop"));
    printf("************************************\nhydro cycle run time= %14.8g us\n"
           "************************************\n", wall);
    if (outbase) {
        char fn[4096];
        snprintf(fn, sizeof(fn), "%s.xy", outbase);
        orc_write_xy(sim, fn);
        orc_write_gold(sim, outbase);
    }
    orc_destroy(sim);
    return 0;
}
