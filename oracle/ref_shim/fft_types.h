/* Stand-in for the Charm-FFT type header that eesDataClass.h includes; the
 * oracle's EES build uses none of its types.  Test infrastructure only. */
