/* Empty: the SPM-internal header bcsc/bvec_zlapmr.c includes; the one routine
 * it needs (spm_get_glob2loc) is declared in spm.h.  Test infrastructure. */
