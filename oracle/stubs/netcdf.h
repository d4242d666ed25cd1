/* Stub for building the reference CPU sources in place: netCDF output is not
 * on the step path and libnetcdf is not installed. TEST INFRASTRUCTURE ONLY. */
