function Fx = apply_adjoint_operator(y, G, Lambda) %#ok<INUSD>
% src/apply_adjoint_operator.m:1 over libfhs_b200: Fx = G' * (Lambda .* y)
% for channel G.channel (0-based) of an fhs_operator handle.
Fx = fhs_mex('apply_adjoint_operator', G.h, G.channel, complex(y(:)));
end
