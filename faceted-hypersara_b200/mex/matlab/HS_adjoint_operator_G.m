function x = HS_adjoint_operator_G(y, G, W, At, N, M, flag_visibility_gridding, Lambda) %#ok<INUSD>
% lib/operators/HS_adjoint_operator_G.m over libfhs_b200 (real part, as the
% solvers use it): y{l}{b} -> x [N, M, L] (the reference's argument order).
x = fhs_mex('HS_adjoint_operator_G', G.h, complex(fhs_cat_blocks(y)), [N, M, numel(y)]);
end
