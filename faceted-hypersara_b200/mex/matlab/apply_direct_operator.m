function y = apply_direct_operator(Fx, G, Lambda) %#ok<INUSD>
% src/apply_direct_operator.m:1 over libfhs_b200: y = Lambda .* (G * Fx) for
% channel G.channel (0-based) of an fhs_operator handle; Lambda lives in a
% visibility-gridding handle (fhs_mex('measop_create_dr', ...)).
y = fhs_mex('apply_direct_operator', G.h, G.channel, complex(Fx(:)));
end
