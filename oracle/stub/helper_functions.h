/* Test infrastructure only: empty stand-in for the CUDA samples header the
 * reference's .cu files include (they use nothing from it). */
