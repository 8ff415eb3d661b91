% build_mex.m - compile the MEX gateways that shadow the reference's hot-path
% .m files.  Run from this folder after building libgbm3d.so
% (python -m gbm3d_b200.build), then put this folder ahead of the
% reference's source/ on the MATLAB path:
%   addpath(fileparts(which('build_mex')), '-begin')
% GNU Octave: mkoctfile --mex -I../../include -L.. -lgbm3d <gateway>.c
here = fileparts(mfilename('fullpath'));
inc = ['-I' fullfile(here, '..', '..', 'include')];
lib = ['-L' fullfile(here, '..')];
gateways = {'matchBlocksCPU', 'denoiseAndAggregateGPU', 'matchBlocksWie', ...
            'denoiseAndAggregateWieFast', 'denoiseAndAggregateWie', 'matchBlocksGPU', ...
            'matchBlocksV', 'denoiseAndAggregateV'};
for k = 1:numel(gateways)
    mex('-outdir', here, inc, lib, '-lgbm3d', fullfile(here, [gateways{k} '.c']));
end
