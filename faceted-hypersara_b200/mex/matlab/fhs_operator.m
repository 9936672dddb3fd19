function G = fhs_operator(M, N, om, weights, blocks, oy, ox, J, device)
% FHS_OPERATOR  Measurement operator over libfhs_b200 (through fhs_mex); it
% stands in for the reference's A, At, G, W of
% lib/operators/util_gen_measurement_operator_synth.m.
%   M, N     image rows and columns
%   om{l}    [v u] frequencies of channel l in radians, one row per visibility
%   weights  cell of per-visibility G row weights (nW), or {} for none
%   blocks{l} block sizes of channel l (at most 16)
%   oy, ox, J, device   oversampling (2, 2), taps (7), CUDA device (0)
if nargin < 6 || isempty(oy), oy = 2; end
if nargin < 7 || isempty(ox), ox = 2; end
if nargin < 8 || isempty(J), J = 7; end
if nargin < 9 || isempty(device), device = 0; end
L = numel(om);
G.h = fhs_mex('measop_create', M, N, oy, ox, J, L, device);
for l = 1:L
    w = [];
    if ~isempty(weights), w = double(weights{l}(:)); end
    fhs_mex('measop_set_channel', G.h, l - 1, double(om{l}(:, 1)), double(om{l}(:, 2)), w, ...
            double(blocks{l}(:)));
end
fhs_mex('measop_commit', G.h);
G.M = M;
G.N = N;
G.L = L;
G.blocks = blocks;
G.channel = 0;
end
