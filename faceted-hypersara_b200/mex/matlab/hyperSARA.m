function xsol = hyperSARA(y, epsilon, A, At, pU, G, W, param, K, ...
    wavelet, nlevel, spectral_chunk, n_channels, M, N, oy, ox, ...
    warmstart_name, checkpoint_name, flag_dimensionality_reduction, Sigma, varargin) %#ok<INUSD>
% src/hs/hyperSARA.m over libfhs_b200 (see facetHyperSARA.m).
cfg = struct('L', numel(y), 'Ny', M, 'Nx', N, 'Qy', 1, 'Qx', 1, 'overlap_y', 0, 'overlap_x', 0, ...
             'nlevel', nlevel, 'n_groups', 1, 'window', 0);
xinit = [];
if ~isempty(varargin), xinit = varargin{1}; end
xsol = fhs_solve('hs', G, y, epsilon, param, cfg, xinit);
end
