/*
 * Stand-in for a project's machine.h (td-project-template/machine.h).  The reference uses it for
 * MPI/GPU placement of its host driver; this library runs one device per process and needs none
 * of it, so the file only has to exist for an unmodified predefines.h to compile.
 */
#ifndef WTD_MACHINE_STUB_H
#define WTD_MACHINE_STUB_H
#ifndef GPUS_PER_NODE
#define GPUS_PER_NODE 1
#endif
#endif
