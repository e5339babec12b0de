/*
 * ref_stubs.c — no-op replacements for the reference's HDF5-backed units
 * (io_xdmf.c, checkpoint.c), which cannot be compiled here because libhdf5
 * is absent.  With these stubs a deck that asks for "DataFormat XDMF" runs
 * its physics unchanged and writes no field files; the XDMF grain
 * renumbering (io_xdmf.c getRenumberArray) therefore draws no rand() values.
 * Restart (-r) is rejected.  Test infrastructure only.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

void xdmf_prepareIO(void) {}
void xdmf_writeMain(void) {}
void xdmf_writeSubblocks(void) {}
void xdmf_closeIO(void) {}

void writeTaskCheckpoint(uint64_t timestep) { (void)timestep; }
void writeMainCheckpoint(void) {}
void clean_checkpoint(void) {}
void mainRestart(uint64_t restart)
{
    (void)restart;
    fprintf(stderr, "mmsref: restart needs HDF5, which is not available\n");
    exit(2);
}
void taskRestart(uint64_t restart) { mainRestart(restart); }
