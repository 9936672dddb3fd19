function p = proj_l2ball(x, eps, y)
% src/proj_l2ball.m over libfhs_b200 (FP64 on the GPU).
p = reshape(fhs_mex('proj_l2ball', complex(x(:)), eps, complex(y(:))), size(x));
end
