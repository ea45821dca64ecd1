// k_step's threads per CTA, one definition for the kernel (both builds) and
// the host code that sizes and launches it; the NVRTC build is also given
// the library's value as -DAQ_CH, so a build option reaches both.
#pragma once

#ifndef AQ_CH
#define AQ_CH 64
#endif
