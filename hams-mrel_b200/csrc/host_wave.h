// host_wave.h -- dispersion roots on the host (host_wave.cpp).
#pragma once

// DISPERSION (WavDynSubs.f90:40-127): the propagating wave number and the
// first nrt-1 evanescent roots for frequency w in depth h, into wvn[0..nrt).
void hams_dispersion(double* wvn, int nrt, double w, double h);
