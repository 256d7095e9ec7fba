/* Empty stand-in for mpi.h: the reference includes it but every MPI call on the
 * single-thread simulator path is an empty stub (GLIFENeurons.cpp:54-60). */
