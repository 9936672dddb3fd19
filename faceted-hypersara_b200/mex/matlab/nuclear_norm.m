function f = nuclear_norm(x)
% src/nuclear_norm.m over libfhs_b200: sum of the singular values of x
% reshaped [M*N, L] (FP64 Gram and eigensolve on the GPU).
f = fhs_mex('nuclear_norm', reshape(double(x), [], size(x, 3)));
end
