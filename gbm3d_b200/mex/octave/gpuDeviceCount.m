function n = gpuDeviceCount()
% Stand-in, for GNU Octave only, for the Parallel Computing Toolbox function
% of the same name: it reports no gpuArray devices.  The reference's
% waveTransforms3D/getWaveFilters3Dbior.m (lines 33-36) calls gpuDeviceCount to
% decide whether to return its filter bank as a gpuArray; Octave has no such
% function, so without this file GBM3D.m stops there.  With it the bank stays a
% host array, which the denoiseAndAggregateGPU gateway takes as is.  Add this
% folder to Octave's path only: on MATLAB's path it would hide the toolbox
% function.
n = 0;
end
