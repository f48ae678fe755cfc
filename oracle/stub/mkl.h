/* Empty stand-in for Intel MKL's header.
 *
 * The reference simulator includes <mkl.h> (shear/src/Parameters.h:19,
 * extensional/src/Parameters.h:19) but calls no MKL routine, so an empty
 * header is enough to compile it with gcc for the test oracle.  Test
 * infrastructure only. */
#ifndef BD_ORACLE_STUB_MKL_H
#define BD_ORACLE_STUB_MKL_H
#endif
