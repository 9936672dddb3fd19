function y = HS_forward_operator_G(x, G, W, A, flag_visibility_gridding, Lambda) %#ok<INUSD>
% lib/operators/HS_forward_operator_G.m over libfhs_b200: x [M, N, L] ->
% y{l}{b}; G is an fhs_operator handle (A, W and Lambda are inside it).
y = fhs_split_blocks(fhs_mex('HS_forward_operator_G', G.h, double(x)), G.blocks);
end
