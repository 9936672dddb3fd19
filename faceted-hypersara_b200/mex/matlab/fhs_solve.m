function xsol = fhs_solve(algo, G, y, epsilon, param, cfg, xinit)
% FHS_SOLVE  Shared body of the solver wrappers: one fhs_mex('solver', ...)
% call (create, set params and data, init, run to the stopping rule, read x).
%   cfg: L, Ny, Nx, Qy, Qx, overlap_y, overlap_x, nlevel, n_groups, window
if nargin < 7, xinit = []; end
if ~isempty(xinit), xinit = double(xinit); end
p = param;
if isfield(p, 'squared_operator_norm') && ~isfield(p, 'nu2')
    p.nu2 = p.squared_operator_norm;
end
xsol = fhs_mex('solver', G.h, algo, cfg, p, complex(fhs_cat_blocks(y)), ...
               double(fhs_cat_blocks(epsilon)), xinit);
end
