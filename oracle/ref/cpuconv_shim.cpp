// C entry points over the upstream RayTraceDicom CPU Gaussian convolution
// (RayTraceDicom-main/src/cpu_convolution_1d.cpp: xConvCpu, yConvCpu), compiled from
// its sources by oracle/ref/build_upstream_conv.sh. Test infrastructure: the bench
// times it as the stage-level CPU baseline of the spot-to-ray convolution.
#include "cpu_convolution_1d.h"

extern "C" {

void upstream_x_conv_cpu(const float* in, float* out, float rSigmaEff, unsigned rad, unsigned inWidth,
                         unsigned outWidth, unsigned height, int inOutOffset) {
    xConvCpu(in, out, rSigmaEff, rad, inWidth, outWidth, height, inOutOffset);
}

void upstream_y_conv_cpu(const float* in, float* out, float rSigmaEff, unsigned rad, unsigned inHeight,
                         unsigned width, int inOutOffset) {
    yConvCpu(in, out, rSigmaEff, rad, inHeight, width, inOutOffset);
}

}  // extern "C"
