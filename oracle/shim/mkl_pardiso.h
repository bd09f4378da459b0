/* Stand-in for mkl_pardiso.h: everything needed is in the shim mkl.h. */
