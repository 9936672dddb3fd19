function xsol = sara(y, epsilon, A, At, pU, G, W, Psi, Psit, param, ...
    warmstart_name, checkpoint_name, alph, ...
    flag_dimensionality_reduction, Lambda, varargin) %#ok<INUSD>
% src/sara/sara.m over libfhs_b200: single-channel SARA (db1..db8 + Dirac,
% 4 levels, in place of Psi / Psit).  varargin{1} = xinit.
cfg = struct('L', numel(y), 'Ny', G.M, 'Nx', G.N, 'Qy', 1, 'Qx', 1, 'overlap_y', 0, 'overlap_x', 0, ...
             'nlevel', 4, 'n_groups', 1, 'window', 0);
xinit = [];
if ~isempty(varargin), xinit = varargin{1}; end
xsol = fhs_solve('sara', G, y, epsilon, param, cfg, xinit);
end
