function f = compute_sara_prior(x, Psit, n_wavelet_coefficients) %#ok<INUSD>
% src/compute_sara_prior.m over libfhs_b200: sum over the SARA coefficients
% of the l2 norm across channels; the dictionary is db1..db8 + Dirac at 4
% levels (imaging/default_parameters.json "sara"), applied on the GPU.
f = fhs_mex('compute_sara_prior', double(x), 4);
end
