/* Stand-ins for the CPU leg of the reference's Hausdorff benchmark
 * (bench/hausdorff_bench.cu declares them; the reference implements them in
 * bench/bench_cpu_hausdorff.cpp on CoACD/src, which the reference tree does
 * not include).  They do no work and return -1, so the benchmark's CPU rows
 * are meaningless and only its GPU rows are read.  Measurement
 * infrastructure only, linked into oracle/_ref/hausdorff_bench. */
double bench_cpu_hausdorff_single(const float* va, const int* ta, int nva, int nta, const float* vb,
                                  const int* tb, int nvb, int ntb, unsigned int resolution, unsigned int seed)
{
    (void)va; (void)ta; (void)nva; (void)nta; (void)vb; (void)tb; (void)nvb; (void)ntb; (void)resolution; (void)seed;
    return -1.0;
}

double bench_cpu_hausdorff_batch(const float* va, const int* ta, int nva, int nta, const float* vb, const int* tb,
                                 int nvb, int ntb, int batch, unsigned int resolution, unsigned int seed)
{
    (void)va; (void)ta; (void)nva; (void)nta; (void)vb; (void)tb; (void)nvb; (void)ntb; (void)batch;
    (void)resolution; (void)seed;
    return -1.0;
}
