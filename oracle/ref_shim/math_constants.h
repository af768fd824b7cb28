/* Empty stand-in for CUDA's math_constants.h: the reference's exp_proj.cu
 * includes it but uses none of its constants (host build, oracle/_ref). */
