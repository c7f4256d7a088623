/*
 * ref_bench.c -- times CM3D's own MD step on the host.  Test and
 * CPU-timing infrastructure only: bench.py's CPU-baseline leg runs it; it is compiled
 * against the reference's headers and linked against the reference's
 * archives (oracle/Makefile), never part of the product.
 *
 * It replays CM3D's start-up exactly as ref_dump.c does (md_startup,
 * readpos, step_init), then times `nsteps` iterations of the loop body of
 * md_mdcntr_new (main/md_mdcntr.new.c:176-178: step, geteng, gettngbr) with
 * CLOCK_MONOTONIC and prints one JSON line:
 *   {"natoms": N, "steps": S, "seconds": T, "atom_steps_per_s": N*S/T,
 *    "poter": U}
 *
 * usage:  ref_bench <cm3d input file> <nsteps> [warmup [trace]]
 *         (run from the deck's directory; warmup: untimed loop iterations
 *         before the timed ones, default 0; trace: after every timed step
 *         print "T istep poth potra zke" at %.17g -- the terms of CM3D's
 *         conserved energy ham of an NVE run, integrate/md_averages.new.c:100)
 */
#include <time.h>

#include "md.h"

int main(int argc, char *argv[])
{
  SIMPARMS simparms;
  FILENAMES filenames;
  COORDS coords;
  SUBSPACE subspace;
  WRITE_STEP write_step;
  NGBR ngbr;
  INTER inter;
  ENERGIES energies;
  int s, nsteps, warmup, trace;
  struct timespec t0, t1;
  double sec;

  if (argc < 3) {
    fprintf(stderr, "usage: %s input nsteps\n", argv[0]);
    return 2;
  }
  nsteps = atoi(argv[2]);
  warmup = argc > 3 ? atoi(argv[3]) : 0;
  trace = argc > 4 && strcmp(argv[4], "trace") == 0;
  memset(&simparms, 0, sizeof simparms);
  memset(&filenames, 0, sizeof filenames);
  memset(&coords, 0, sizeof coords);
  memset(&subspace, 0, sizeof subspace);
  memset(&write_step, 0, sizeof write_step);
  memset(&ngbr, 0, sizeof ngbr);
  memset(&inter, 0, sizeof inter);
  memset(&energies, 0, sizeof energies);
  simparms.rank = 0;
  simparms.size = 1;
  strcpy(filenames.infile, argv[1]);
  strcpy(filenames.command, argv[0]);
  md_startup(&filenames, &simparms, &subspace, &write_step, &inter, &ngbr, &coords);
  readpos(argv[0], filenames.initfile, &simparms, &energies.estep, &energies, &coords);
  if (simparms.istart == 1) {
    samvel(&simparms, &coords, 1);
    samveta(&simparms, &coords);
  }
  zero_averages(&simparms, &energies);
  gethinv9(coords.hmat, coords.hmati);
  step_init(&simparms, &coords, &energies, &inter, &ngbr);
  simparms.istep = 1;
  for (s = 0; s < warmup; s++, simparms.istep++) {
    step(&simparms, &coords, &energies, &inter, &ngbr);
    geteng(&simparms, &coords, &energies);
    gettngbr(&ngbr);
  }
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (s = 0; s < nsteps; s++, simparms.istep++) {
    step(&simparms, &coords, &energies, &inter, &ngbr);
    geteng(&simparms, &coords, &energies);
    gettngbr(&ngbr);
    if (trace)
      printf("T %d %.17g %.17g %.17g\n", simparms.istep, energies.poth, energies.potra, energies.zke);
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  sec = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
  printf("{\"natoms\": %d, \"steps\": %d, \"seconds\": %.9g, \"atom_steps_per_s\": %.9g, "
         "\"poter\": %.17g}\n",
         simparms.natoms, nsteps, sec, sec > 0 ? simparms.natoms * (double)nsteps / sec : 0.0,
         energies.poter);
  return 0;
}
