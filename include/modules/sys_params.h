#ifndef SYSPARAMS_H
#define SYSPARAMS_H

#ifndef __CUDACC__
#ifndef __device__
#define __device__
#endif
#endif

namespace sys_params {
    __device__ constexpr int particlesNumber = 8;
    __device__ constexpr int inverseFilling = 3;

    __device__ constexpr int confinementExponent = 2;
    __device__ constexpr float confinementStrength = 1;
    __device__ constexpr double confinementOmega = 0.01;
    __device__ constexpr double confinementKappa = 0.0001;

    __device__ constexpr float RCl = 6.9282032302755088;
    __device__ constexpr float DCl = 13.856406460551018;
    __device__ constexpr float RCl_reciprocal = 0.14433756729740646;
    __device__ constexpr float R0_reciprocal = 0.28867513459481292;

    __device__ constexpr int ansatzExtendedMaxDegree = 25;
    __device__ constexpr int ansatzMaxPartitionSize = 8;
    __device__ constexpr int ansatzSubspaceDimension = 4096;

    __device__ constexpr int ansatzMultipletSize = 8;

    __device__ constexpr int ansatzMaxAngularMomentum = 15;
    __device__ constexpr int angularMomentumCutoff = 36;

}

#endif
