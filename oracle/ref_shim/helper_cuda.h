/* Empty stand-in for the CUDA samples header that the reference's Boussinesq
 * sources include (3D_Boussinesq/src/cuda.cu:11); none of its helpers is used. */
